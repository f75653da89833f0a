// C ABI of libautorift_gpu: contexts, device-resident image pairs and the track entry points.
// Declared in include/autorift_gpu.h, where each entry point cites the reference interface it
// replaces.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ar_internal.cuh"

namespace {

// Host threads that split large copies between caller-owned (pageable) arrays and the pinned
// staging buffers. One core copies at roughly a fifth of what the PCIe link carries, so a
// single-threaded copy, not the DMA, set the pace of uploads. A copy is cut into pieces that
// the calling thread and the workers claim from one counter; the counter carries the copy's
// generation in its upper half, so a worker that wakes late can never claim a piece of a
// later copy with an earlier copy's pointers. One pool serves every context of the process and
// runs one copy at a time: the host's memory bandwidth is the shared resource, and the serving
// slots' contexts copying at once with a pool each oversubscribed the cores (three slots ran
// slower than one pair at a time).
class CopyPool {
public:
    explicit CopyPool(int workers) {
        for (int i = 0; i < workers; ++i) threads_.emplace_back([this] { work(); });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_job_.notify_all();
        for (auto& t : threads_) t.join();
    }
    // memcpy(dst, src, bytes), shared with the workers when it is large; callers from several
    // contexts take turns.
    void copy(void* dst, const void* src, size_t bytes) {
        constexpr size_t kMinSplit = 512u << 10, kPieceAlign = 64u << 10;
        if (threads_.empty() || bytes < kMinSplit) {
            std::memcpy(dst, src, bytes);
            return;
        }
        std::lock_guard<std::mutex> turn(turn_mu_);
        const size_t ways = threads_.size() + 1;
        Job j;
        j.dst = static_cast<unsigned char*>(dst);
        j.src = static_cast<const unsigned char*>(src);
        j.bytes = bytes;
        j.piece = (bytes / ways + kPieceAlign - 1) / kPieceAlign * kPieceAlign;
        j.parts = static_cast<uint32_t>((bytes + j.piece - 1) / j.piece);
        {
            std::lock_guard<std::mutex> lk(mu_);
            j.gen = ++gen_;
            job_ = j;
            done_ = 0;
            next_.store(static_cast<uint64_t>(j.gen) << 32);
        }
        cv_job_.notify_all();
        run(j);
        std::unique_lock<std::mutex> lk(mu_);
        cv_done_.wait(lk, [&] { return done_ == j.parts; });
    }

private:
    struct Job {
        unsigned char* dst = nullptr;
        const unsigned char* src = nullptr;
        size_t bytes = 0, piece = 0;
        uint32_t parts = 0, gen = 0;
    };
    void run(const Job& j) {
        uint32_t mine = 0;
        uint64_t cur = next_.load();
        while ((cur >> 32) == j.gen && static_cast<uint32_t>(cur) < j.parts) {
            if (!next_.compare_exchange_weak(cur, cur + 1)) continue;
            const size_t off = static_cast<size_t>(static_cast<uint32_t>(cur)) * j.piece;
            std::memcpy(j.dst + off, j.src + off, std::min(j.piece, j.bytes - off));
            ++mine;
            cur = next_.load();
        }
        if (mine) {
            std::lock_guard<std::mutex> lk(mu_);
            if (gen_ == j.gen) done_ += mine;
            if (done_ == j.parts) cv_done_.notify_all();
        }
    }
    void work() {
        uint32_t seen = 0;
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_job_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                j = job_;
            }
            run(j);
        }
    }
    std::vector<std::thread> threads_;
    std::mutex turn_mu_;  // one copy at a time
    std::mutex mu_;
    std::condition_variable cv_job_, cv_done_;
    Job job_;
    uint32_t gen_ = 0, done_ = 0;
    std::atomic<uint64_t> next_{0};
    bool stop_ = false;
};

int copy_workers() {
    const unsigned hw = std::thread::hardware_concurrency();
    return static_cast<int>(std::min(15u, hw > 1 ? hw - 1 : 0u));
}

// The process's copy pool, created by the first context that stages a copy and released with
// the last one.
std::shared_ptr<CopyPool> shared_copy_pool() {
    static std::mutex m;
    static std::weak_ptr<CopyPool> pool;
    std::lock_guard<std::mutex> lk(m);
    std::shared_ptr<CopyPool> p = pool.lock();
    if (!p) {
        p = std::make_shared<CopyPool>(copy_workers());
        pool = p;
    }
    return p;
}

}  // namespace

struct ar_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    std::string err;
    std::mutex mu;  // one call at a time per context
    ar::TrackScratch scratch;
    // Pinned staging for host<->device copies of caller-owned (pageable) arrays.
    unsigned char* pinned = nullptr;
    size_t pinned_bytes = 0;
    cudaEvent_t staged[2] = {nullptr, nullptr};
    std::shared_ptr<CopyPool> copier;  // the process's host threads for the staging copies
    // Device buffers for host point sets and outputs, grown on demand.
    void* dbuf = nullptr;
    size_t dbuf_bytes = 0;
    // Scratch of the multichip search, grown on demand and kept between calls.
    void* arena = nullptr;
    size_t arena_bytes = 0;
    // Stream-ordered pool for pair images and per-call scratch: freed blocks stay with the
    // context and are reused without a device-wide synchronisation.
    cudaMemPool_t pool = nullptr;
    // The request loop, started by the first ar_submit.
    std::mutex serve_mu;
    ar::ServeEngine* serve = nullptr;
    int serve_slots = 4;
    size_t serve_budget = 0;
};

struct ar_pair {
    ar_ctx* ctx = nullptr;
    int dtype = 0;
    int64_t nrows = 0, ncols = 0;
    void* ref = nullptr;
    void* sec = nullptr;
    uint8_t* ref_valid = nullptr;
    uint8_t* sec_valid = nullptr;
    uint8_t* valid = nullptr;  // ref_valid .& sec_valid
    // Recorded on the context stream when the pair's contents are complete (the upload or the
    // preparation is queued, not awaited); work on another stream waits for it.
    cudaEvent_t ready = nullptr;
};

namespace {

constexpr size_t kStageBytes = 32u << 20;  // two halves of 16 MiB

size_t elem_size(int dtype) {
    switch (dtype) {
        case AR_U8: return 1;
        case AR_U16: return 2;
        case AR_I16: return 2;
        case AR_F32: return 4;
        case AR_F64: return 8;
        default: return 0;
    }
}

int fail(ar_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_fail(ar_ctx* ctx, cudaError_t e, const char* what) {
    const int code = e == cudaErrorMemoryAllocation ? AR_ERR_OOM : AR_ERR_CUDA;
    return fail(ctx, code, std::string(what) + ": " + cudaGetErrorString(e));
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

cudaError_t ensure_pinned(ar_ctx* c) {
    if (c->pinned) return cudaSuccess;
    cudaError_t e = cudaMallocHost(&c->pinned, kStageBytes);
    if (e != cudaSuccess) return e;
    c->pinned_bytes = kStageBytes;
    c->copier = shared_copy_pool();
    for (auto& ev : c->staged) {
        e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Host (pageable) -> device through the two pinned halves, so the CPU copy of one chunk
// overlaps the DMA of the previous one. Stream-ordered; returns once all chunks are queued.
cudaError_t stage_h2d(ar_ctx* c, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return cudaSuccess;
    cudaError_t e = ensure_pinned(c);
    if (e != cudaSuccess) return e;
    const size_t half = c->pinned_bytes / 2;
    size_t off = 0;
    int slot = 0;
    while (off < bytes) {
        const size_t n = std::min(half, bytes - off);
        e = cudaEventSynchronize(c->staged[slot]);  // the slot's previous DMA has finished
        if (e != cudaSuccess) return e;
        unsigned char* buf = c->pinned + slot * half;
        c->copier->copy(buf, static_cast<const unsigned char*>(src) + off, n);
        e = cudaMemcpyAsync(static_cast<unsigned char*>(dst) + off, buf, n, cudaMemcpyHostToDevice,
                            c->stream);
        if (e != cudaSuccess) return e;
        e = cudaEventRecord(c->staged[slot], c->stream);
        if (e != cudaSuccess) return e;
        off += n;
        slot ^= 1;
    }
    return cudaSuccess;
}

// Device -> host (pageable) through the pinned halves; synchronous.
cudaError_t stage_d2h(ar_ctx* c, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return cudaSuccess;
    cudaError_t e = ensure_pinned(c);
    if (e != cudaSuccess) return e;
    const size_t half = c->pinned_bytes / 2;
    size_t off = 0;
    int slot = 0;
    size_t pending_off[2] = {0, 0}, pending_n[2] = {0, 0};
    while (off < bytes || pending_n[0] || pending_n[1]) {
        if (off < bytes) {
            e = cudaEventSynchronize(c->staged[slot]);
            if (e != cudaSuccess) return e;
            if (pending_n[slot]) {
                c->copier->copy(static_cast<unsigned char*>(dst) + pending_off[slot],
                                c->pinned + slot * half, pending_n[slot]);
                pending_n[slot] = 0;
            }
            const size_t n = std::min(half, bytes - off);
            e = cudaMemcpyAsync(c->pinned + slot * half, static_cast<const unsigned char*>(src) + off,
                                n, cudaMemcpyDeviceToHost, c->stream);
            if (e != cudaSuccess) return e;
            e = cudaEventRecord(c->staged[slot], c->stream);
            if (e != cudaSuccess) return e;
            pending_off[slot] = off;
            pending_n[slot] = n;
            off += n;
            slot ^= 1;
        } else {
            for (int s = 0; s < 2; ++s) {
                if (!pending_n[s]) continue;
                e = cudaEventSynchronize(c->staged[s]);
                if (e != cudaSuccess) return e;
                c->copier->copy(static_cast<unsigned char*>(dst) + pending_off[s],
                                c->pinned + s * half, pending_n[s]);
                pending_n[s] = 0;
            }
        }
    }
    return cudaSuccess;
}

cudaError_t ensure_dbuf(ar_ctx* c, size_t bytes) {
    if (c->dbuf_bytes >= bytes) return cudaSuccess;
    // Stream-ordered on the context stream (the only one that uses these buffers).
    if (c->dbuf) cudaFreeAsync(c->dbuf, c->stream);
    c->dbuf = nullptr;
    c->dbuf_bytes = 0;
    cudaError_t e = cudaMallocFromPoolAsync(&c->dbuf, bytes, c->pool, c->stream);
    if (e != cudaSuccess) return e;
    c->dbuf_bytes = bytes;
    return cudaSuccess;
}

// Per-image masks (given ones normalised to 0/1, missing ones from finiteness, the ImagePair
// default of src/preprocess.jl:74-79) and their intersection, valid(pair).
template <typename T>
__global__ void k_make_valid(const T* ref, const T* sec, uint8_t* rv, uint8_t* sv, bool have_rv,
                             bool have_sv, uint8_t* out, int64_t n) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const bool a = have_rv ? rv[i] != 0 : isfinite(static_cast<double>(ref[i]));
    const bool b = have_sv ? sv[i] != 0 : isfinite(static_cast<double>(sec[i]));
    rv[i] = a ? 1 : 0;
    sv[i] = b ? 1 : 0;
    out[i] = (a && b) ? 1 : 0;
}

__global__ void k_and_masks(const uint8_t* a, const uint8_t* b, uint8_t* out, int64_t n) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i < n) out[i] = (a[i] && b[i]) ? 1 : 0;
}

template <typename T>
cudaError_t launch_make_valid(ar_pair* p, bool have_rv, bool have_sv, cudaStream_t s) {
    const int threads = 256;
    const int64_t n = p->nrows * p->ncols;
    k_make_valid<T><<<static_cast<unsigned>((n + threads - 1) / threads), threads, 0, s>>>(
        static_cast<const T*>(p->ref), static_cast<const T*>(p->sec), p->ref_valid, p->sec_valid,
        have_rv, have_sv, p->valid, n);
    return cudaGetLastError();
}

bool is_pow2(int v) { return v >= 1 && (v & (v - 1)) == 0; }

// Pool allocations, ordered on the context stream.
cudaError_t dalloc(ar_ctx* c, void** p, size_t bytes) {
    *p = nullptr;
    return cudaMallocFromPoolAsync(p, std::max<size_t>(bytes, 256), c->pool, c->stream);
}
template <typename T>
cudaError_t dalloc(ar_ctx* c, T** p, size_t bytes) {
    void* q = nullptr;
    cudaError_t e = dalloc(c, &q, bytes);
    *p = static_cast<T*>(q);
    return e;
}
void dfree(ar_ctx* c, void* p) {
    if (p) cudaFreeAsync(p, c->stream);
}
void pair_free(ar_pair* p) {
    dfree(p->ctx, p->ref);
    dfree(p->ctx, p->sec);
    dfree(p->ctx, p->valid);
    p->ref = p->sec = nullptr;
    p->valid = p->ref_valid = p->sec_valid = nullptr;
    if (p->ready) cudaEventDestroy(p->ready);
    p->ready = nullptr;
}

// Marks the pair complete on the context stream (its upload or preparation queued there).
cudaError_t pair_mark_ready(ar_ctx* c, ar_pair* p) {
    if (!p->ready) {
        cudaError_t e = cudaEventCreateWithFlags(&p->ready, cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
    }
    return cudaEventRecord(p->ready, c->stream);
}

// Orders work about to be queued on `s` after the pair's contents are complete.
cudaError_t pair_wait(ar_ctx* c, const ar_pair* p, cudaStream_t s) {
    if (s == c->stream || !p->ready) return cudaSuccess;
    return cudaStreamWaitEvent(s, p->ready, 0);
}

}  // namespace

extern "C" {

int ar_version(void) { return 100; }

int ar_ctx_create(int device, ar_ctx** out) {
    if (!out) return AR_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return AR_ERR_ARG;
    DeviceGuard g(device);
    ar_ctx* c = new ar_ctx();
    c->device = device;
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        e = cudaMemPoolCreate(&c->pool, &props);
    }
    if (e == cudaSuccess) {
        uint64_t keep = UINT64_MAX;  // never trim: the context reuses what it frees
        e = cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e != cudaSuccess) {
        if (c->pool) cudaMemPoolDestroy(c->pool);
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
        return AR_ERR_CUDA;
    }
    c->scratch.pool = c->pool;
    *out = c;
    return AR_OK;
}

int ar_ctx_destroy(ar_ctx* c) {
    if (!c) return AR_ERR_ARG;
    {
        std::lock_guard<std::mutex> lk(c->serve_mu);
        ar::serve_destroy(c->serve);  // completes every queued request first
        c->serve = nullptr;
    }
    {
        DeviceGuard g(c->device);
        std::lock_guard<std::mutex> lk(c->mu);
        cudaStreamSynchronize(c->stream);
        cudaFree(c->scratch.sub_count);
        cudaFree(c->scratch.sub_point);
        cudaFree(c->scratch.sub_origin);
        cudaFree(c->scratch.sub_patch);
        cudaFree(c->scratch.geom);
        cudaFree(c->scratch.status);
        for (auto& r : c->scratch.timer.recs)
            for (auto ev : r) c->scratch.timer.pool.push_back(ev);
        for (auto ev : c->scratch.timer.pool) cudaEventDestroy(ev);
        cudaFree(c->scratch.timer.flops);
        if (c->scratch.done) cudaEventDestroy(c->scratch.done);
        for (auto ev : c->scratch.tune_ev)
            if (ev) cudaEventDestroy(ev);
        cudaFree(c->dbuf);
        cudaFree(c->arena);
        if (c->pinned) cudaFreeHost(c->pinned);
        for (auto& ev : c->staged)
            if (ev) cudaEventDestroy(ev);
        cudaStreamSynchronize(c->stream);
        cudaMemPoolDestroy(c->pool);
        cudaStreamDestroy(c->stream);
    }
    delete c;
    return AR_OK;
}

int ar_last_error(const ar_ctx* c, char* buf, size_t size) {
    if (!c || !buf || size == 0) return AR_ERR_ARG;
    const size_t n = std::min(size - 1, c->err.size());
    std::memcpy(buf, c->err.data(), n);
    buf[n] = '\0';
    return AR_OK;
}

int ar_pair_upload(ar_ctx* c, const void* ref, const void* sec, const uint8_t* ref_valid,
                   const uint8_t* sec_valid, int64_t nrows, int64_t ncols, int dtype,
                   ar_pair** out) {
    if (!c || !ref || !sec || !out) return fail(c, AR_ERR_ARG, "null argument");
    *out = nullptr;
    if (nrows <= 0 || ncols <= 0) return fail(c, AR_ERR_SIZE, "image extents must be positive");
    const size_t es = elem_size(dtype);
    if (es == 0 || dtype == AR_F64) return fail(c, AR_ERR_UNSUPPORTED, "unsupported element type");
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    const int64_t n = nrows * ncols;
    ar_pair* p = new ar_pair();
    p->ctx = c;
    p->dtype = dtype;
    p->nrows = nrows;
    p->ncols = ncols;
    cudaError_t e = dalloc(c, &p->ref, n * es);
    if (e == cudaSuccess) e = dalloc(c, &p->sec, n * es);
    if (e == cudaSuccess) e = dalloc(c, &p->valid, 3 * n);
    if (e == cudaSuccess) {
        p->ref_valid = p->valid + n;
        p->sec_valid = p->valid + 2 * n;
    }
    if (e == cudaSuccess) e = stage_h2d(c, p->ref, ref, n * es);
    if (e == cudaSuccess) e = stage_h2d(c, p->sec, sec, n * es);
    if (e == cudaSuccess && ref_valid) e = stage_h2d(c, p->ref_valid, ref_valid, n);
    if (e == cudaSuccess && sec_valid) e = stage_h2d(c, p->sec_valid, sec_valid, n);
    if (e == cudaSuccess) {
        switch (dtype) {
            case AR_U8: e = launch_make_valid<uint8_t>(p, ref_valid != nullptr, sec_valid != nullptr, c->stream); break;
            case AR_U16: e = launch_make_valid<uint16_t>(p, ref_valid != nullptr, sec_valid != nullptr, c->stream); break;
            case AR_I16: e = launch_make_valid<int16_t>(p, ref_valid != nullptr, sec_valid != nullptr, c->stream); break;
            case AR_F32: e = launch_make_valid<float>(p, ref_valid != nullptr, sec_valid != nullptr, c->stream); break;
        }
    }
    // The caller's arrays are copied into the staging buffers by now; the transfers and the
    // mask kernel complete in stream order (later calls on other streams wait for `ready`).
    if (e == cudaSuccess) e = pair_mark_ready(c, p);
    if (e != cudaSuccess) {
        pair_free(p);
        delete p;
        return cuda_fail(c, e, "ar_pair_upload");
    }
    *out = p;
    return AR_OK;
}

int ar_pair_destroy(ar_pair* p) {
    if (!p) return AR_ERR_ARG;
    {
        DeviceGuard g(p->ctx->device);
        std::lock_guard<std::mutex> lk(p->ctx->mu);
        // The library's own work on the pair is ordered before the frees on the context
        // stream; work the caller queued on its own streams must have completed.
        if (p->ctx->scratch.done) cudaStreamWaitEvent(p->ctx->stream, p->ctx->scratch.done, 0);
        pair_free(p);
    }
    delete p;
    return AR_OK;
}

int ar_pair_info(const ar_pair* p, int* dtype, int64_t* nrows, int64_t* ncols) {
    if (!p) return AR_ERR_ARG;
    if (dtype) *dtype = p->dtype;
    if (nrows) *nrows = p->nrows;
    if (ncols) *ncols = p->ncols;
    return AR_OK;
}

static int check_track_args(ar_ctx* c, const ar_pair* p, const ar_points* pts, int up, int measure) {
    if (!c || !p || !pts) return fail(c, AR_ERR_ARG, "null argument");
    if (p->ctx != c) return fail(c, AR_ERR_ARG, "the pair belongs to another context");
    if (pts->n < 0) return fail(c, AR_ERR_SIZE, "negative point count");
    if (pts->n > 0 && (!pts->x || !pts->y || !pts->radius_x || !pts->radius_y || !pts->dx_prior ||
                       !pts->dy_prior || !pts->chip_size_x || !pts->chip_size_y))
        return fail(c, AR_ERR_ARG, "null point-set field");
    if (!is_pow2(up) || up > 128)
        return fail(c, AR_ERR_ARG, "`upsampling` must be 1 or a power of 2 up to 128");
    if (measure != AR_ZNCC && measure != AR_NCC) return fail(c, AR_ERR_ARG, "unknown measure");
    return AR_OK;
}

namespace {

int track_host(ar_ctx* c, const ar_pair* p, const ar_points* pts, int up, int measure,
               const ar::Rotation* rot, float* dx, float* dy, float* corr, uint8_t* searched);

}  // namespace

int ar_track(ar_ctx* c, const ar_pair* p, const ar_points* pts, int up, int measure, float* dx,
             float* dy, float* corr, uint8_t* searched) {
    return track_host(c, p, pts, up, measure, nullptr, dx, dy, corr, searched);
}

int ar_track_rotated(ar_ctx* c, const ar_pair* p, const ar_points* pts, int up, int measure,
                     const double* angles, int count, float* dx, float* dy, float* corr,
                     uint8_t* searched) {
    if (count == 0) return track_host(c, p, pts, up, measure, nullptr, dx, dy, corr, searched);
    ar::Rotation rot;
    std::string err;
    if (!ar::make_rotation(angles, count, &rot, &err)) return fail(c, AR_ERR_ARG, err);
    return track_host(c, p, pts, up, measure, &rot, dx, dy, corr, searched);
}

}  // extern "C"

namespace {

int track_host(ar_ctx* c, const ar_pair* p, const ar_points* pts, int up, int measure,
               const ar::Rotation* rot, float* dx, float* dy, float* corr, uint8_t* searched) {
    int rc = check_track_args(c, p, pts, up, measure);
    if (rc != AR_OK) return rc;
    const int64_t n = pts->n;
    if (n > 0 && (!dx || !dy || !corr || !searched)) return fail(c, AR_ERR_ARG, "null output");
    if (n == 0) return AR_OK;
    for (int64_t k = 0; k < n; ++k) {
        if (!std::isfinite(pts->x[k]) || !std::isfinite(pts->y[k]) ||
            !std::isfinite(pts->dx_prior[k]) || !std::isfinite(pts->dy_prior[k]))
            return fail(c, AR_ERR_ARG, "point coordinates and priors must be finite");
    }
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    const ar::PassGeometry geom = ar::pass_geometry_host(*pts, p->nrows, p->ncols);
    // One device block: 4 f64 + 4 i64 fields, then the outputs.
    const size_t fb = static_cast<size_t>(n) * 8;
    const size_t need = 8 * fb + 3 * static_cast<size_t>(n) * 4 + static_cast<size_t>(n) + 64;
    cudaError_t e = ensure_dbuf(c, need);
    if (e != cudaSuccess) return cuda_fail(c, e, "ar_track: device buffers");
    unsigned char* base = static_cast<unsigned char*>(c->dbuf);
    ar::DevPoints dp;
    dp.x = reinterpret_cast<const double*>(base + 0 * fb);
    dp.y = reinterpret_cast<const double*>(base + 1 * fb);
    dp.rx = reinterpret_cast<const int64_t*>(base + 2 * fb);
    dp.ry = reinterpret_cast<const int64_t*>(base + 3 * fb);
    dp.dx0 = reinterpret_cast<const double*>(base + 4 * fb);
    dp.dy0 = reinterpret_cast<const double*>(base + 5 * fb);
    dp.csx = reinterpret_cast<const int64_t*>(base + 6 * fb);
    dp.csy = reinterpret_cast<const int64_t*>(base + 7 * fb);
    dp.n = n;
    ar::DevOutputs dout;
    dout.dx = reinterpret_cast<float*>(base + 8 * fb);
    dout.dy = dout.dx + n;
    dout.corr = dout.dy + n;
    dout.searched = reinterpret_cast<uint8_t*>(dout.corr + n);
    const void* srcs[8] = {pts->x, pts->y, pts->radius_x, pts->radius_y,
                           pts->dx_prior, pts->dy_prior, pts->chip_size_x, pts->chip_size_y};
    for (int f = 0; f < 8 && e == cudaSuccess; ++f) e = stage_h2d(c, base + f * fb, srcs[f], fb);
    if (e != cudaSuccess) return cuda_fail(c, e, "ar_track: upload points");
    std::string err;
    e = ar::launch_track(p->dtype, p->ref, p->sec, p->valid, p->nrows, p->ncols, dp, geom, up,
                         measure, dout, c->scratch, c->num_sms, c->stream, &err, nullptr, rot);
    if (e != cudaSuccess)
        return err.empty() ? cuda_fail(c, e, "ar_track") : fail(c, AR_ERR_UNSUPPORTED, err);
    // The three float outputs are contiguous on the device, as is `searched`.
    std::vector<float> tmp;
    e = stage_d2h(c, dx, dout.dx, n * 4);
    if (e == cudaSuccess) e = stage_d2h(c, dy, dout.dy, n * 4);
    if (e == cudaSuccess) e = stage_d2h(c, corr, dout.corr, n * 4);
    if (e == cudaSuccess) e = stage_d2h(c, searched, dout.searched, n);
    if (e != cudaSuccess) return cuda_fail(c, e, "ar_track: download results");
    int st = 0;
    e = ar::read_status(c->scratch, c->stream, &st);
    if (e != cudaSuccess) return cuda_fail(c, e, "ar_track: status");
    if (st) return fail(c, AR_ERR_TIMEOUT, "ar_track: a device wait ran out; results incomplete");
    return AR_OK;
}

}  // namespace

extern "C" {

namespace {

int track_device(ar_ctx* c, const ar_pair* p, const ar_points* pts, int up, int measure,
                 const ar::Rotation* rot, float* dx, float* dy, float* corr, uint8_t* searched,
                 void* stream);

}  // namespace

int ar_track_device(ar_ctx* c, const ar_pair* p, const ar_points* pts, int up, int measure,
                    float* dx, float* dy, float* corr, uint8_t* searched, void* stream) {
    return track_device(c, p, pts, up, measure, nullptr, dx, dy, corr, searched, stream);
}

int ar_track_device_rotated(ar_ctx* c, const ar_pair* p, const ar_points* pts, int up,
                            int measure, const double* angles, int count, float* dx, float* dy,
                            float* corr, uint8_t* searched, void* stream) {
    if (count == 0)
        return track_device(c, p, pts, up, measure, nullptr, dx, dy, corr, searched, stream);
    ar::Rotation rot;
    std::string err;
    if (!ar::make_rotation(angles, count, &rot, &err)) return fail(c, AR_ERR_ARG, err);
    return track_device(c, p, pts, up, measure, &rot, dx, dy, corr, searched, stream);
}

}  // extern "C"

namespace {

int track_device(ar_ctx* c, const ar_pair* p, const ar_points* pts, int up, int measure,
                 const ar::Rotation* rot, float* dx, float* dy, float* corr, uint8_t* searched,
                 void* stream) {
    int rc = check_track_args(c, p, pts, up, measure);
    if (rc != AR_OK) return rc;
    const int64_t n = pts->n;
    if (n > 0 && (!dx || !dy || !corr || !searched)) return fail(c, AR_ERR_ARG, "null output");
    if (n == 0) return AR_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    ar::DevPoints dp{pts->x, pts->y, pts->radius_x, pts->radius_y, pts->dx_prior,
                     pts->dy_prior, pts->chip_size_x, pts->chip_size_y, n};
    ar::PassGeometry geom;
    cudaError_t e = pair_wait(c, p, s);
    if (e != cudaSuccess) return cuda_fail(c, e, "ar_track_device: pair");
    e = ar::pass_geometry_device(dp, p->nrows, p->ncols, c->scratch, s, &geom);
    if (e != cudaSuccess) return cuda_fail(c, e, "ar_track_device: pass geometry");
    ar::DevOutputs dout{dx, dy, corr, searched};
    std::string err;
    e = ar::launch_track(p->dtype, p->ref, p->sec, p->valid, p->nrows, p->ncols, dp, geom, up,
                         measure, dout, c->scratch, c->num_sms, s, &err, nullptr, rot);
    if (e != cudaSuccess)
        return err.empty() ? cuda_fail(c, e, "ar_track_device") : fail(c, AR_ERR_UNSUPPORTED, err);
    return AR_OK;
}

}  // namespace

extern "C" {

int ar_correlate(ar_ctx* c, const void* search, const void* chip, int dtype, int64_t ch,
                 int64_t cw, int64_t rx, int64_t ry, int measure, float* surface,
                 int* degenerate) {
    if (!c || !search || !chip || !surface) return fail(c, AR_ERR_ARG, "null argument");
    if (ch <= 0 || cw <= 0 || rx <= 0 || ry <= 0 || (ch & 1) || (cw & 1))
        return fail(c, AR_ERR_SIZE, "chip extents must be positive and even, radii positive");
    if (measure != AR_ZNCC && measure != AR_NCC) return fail(c, AR_ERR_ARG, "unknown measure");
    const size_t es = elem_size(dtype);
    if (es == 0 || dtype == AR_F64) return fail(c, AR_ERR_UNSUPPORTED, "unsupported element type");
    // One point on a pair whose reference is the search window and whose secondary holds the
    // chip at the window's zero-displacement position. The point sits at 1-based
    // (ry + ch/2 + 0.5, rx + cw/2 + 0.5): after the grid loop's +0.5 shift its window starts
    // at row 1, column 1 and its chip at row ry + 1, column rx + 1 (src/points.jl:358-395).
    const int64_t wr = ch + 2 * ry - 1, wc = cw + 2 * rx - 1;
    std::vector<unsigned char> secimg(static_cast<size_t>(wr * wc) * es, 0);
    const unsigned char* cp = static_cast<const unsigned char*>(chip);
    for (int64_t j = 0; j < cw; ++j)
        std::memcpy(secimg.data() + (ry + (rx + j) * wr) * es, cp + j * ch * es, ch * es);
    std::vector<uint8_t> mask(static_cast<size_t>(wr * wc), 1);
    ar_pair* pair = nullptr;
    int rc = ar_pair_upload(c, search, secimg.data(), mask.data(), mask.data(), wr, wc, dtype, &pair);
    if (rc != AR_OK) return rc;
    const double x = static_cast<double>(rx + cw / 2) + 0.5;
    const double y = static_cast<double>(ry + ch / 2) + 0.5;
    const int64_t rxx = rx, ryy = ry, csx = cw, csy = ch;
    const double zero = 0.0;
    ar_points pts{&x, &y, &rxx, &ryy, &zero, &zero, &csx, &csy, 1};
    {
        std::lock_guard<std::mutex> lk(c->mu);
        DeviceGuard g(c->device);
        const ar::PassGeometry geom = ar::pass_geometry_host(pts, wr, wc);
        const int64_t ns = 2 * ry * 2 * rx;
        cudaError_t e = ensure_dbuf(c, 8 * 8 + 16 + static_cast<size_t>(ns) * 4 + 256);
        unsigned char* base = static_cast<unsigned char*>(c->dbuf);
        double* dd = reinterpret_cast<double*>(base);
        int64_t* di = reinterpret_cast<int64_t*>(base);
        const double hostd[8] = {x, y, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        const int64_t hosti[4] = {rxx, ryy, csx, csy};
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dd, hostd, sizeof(hostd), cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(di + 8, hosti, sizeof(hosti), cudaMemcpyHostToDevice, c->stream);
        ar::DevPoints dp{dd + 0, dd + 1, di + 8, di + 9, dd + 2, dd + 3, di + 10, di + 11, 1};
        float* fo = reinterpret_cast<float*>(base + 128);
        ar::DevOutputs dout{fo, fo + 1, fo + 2, reinterpret_cast<uint8_t*>(fo + 3)};
        float* dsurf = reinterpret_cast<float*>(base + 256);
        if (e == cudaSuccess) e = cudaMemsetAsync(dsurf, 0, ns * 4, c->stream);
        std::string err;
        if (e == cudaSuccess)
            e = ar::launch_track(dtype, pair->ref, pair->sec, pair->valid, wr, wc, dp, geom, 1,
                                 measure, dout, c->scratch, c->num_sms, c->stream, &err, dsurf);
        float outs[4];
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(outs, fo, sizeof(outs), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = stage_d2h(c, surface, dsurf, ns * 4);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) {
            rc = err.empty() ? cuda_fail(c, e, "ar_correlate") : fail(c, AR_ERR_UNSUPPORTED, err);
        } else {
            uint8_t sr;
            std::memcpy(&sr, &outs[3], 1);
            if (degenerate) *degenerate = (sr && std::isnan(outs[2])) ? 1 : 0;
        }
    }
    ar_pair_destroy(pair);
    return rc;
}

int ar_refine_patches(ar_ctx* c, const float* patches, int64_t count, int up, int32_t* row,
                      int32_t* col, float* value) {
    if (!c || (count > 0 && (!patches || !row || !col || !value)))
        return fail(c, AR_ERR_ARG, "null argument");
    if (!is_pow2(up) || up < 2 || up > 128)
        return fail(c, AR_ERR_ARG, "`upsampling` must be a power of 2 in [2, 128]");
    if (count <= 0) return AR_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    const size_t need = static_cast<size_t>(count) * (25 * 4 + 4 + 4 + 4) + 64;
    cudaError_t e = ensure_dbuf(c, need);
    if (e != cudaSuccess) return cuda_fail(c, e, "ar_refine_patches: device buffers");
    float* dpatch = static_cast<float*>(c->dbuf);
    int32_t* drow = reinterpret_cast<int32_t*>(dpatch + count * 25);
    int32_t* dcol = drow + count;
    float* dval = reinterpret_cast<float*>(dcol + count);
    e = stage_h2d(c, dpatch, patches, count * 25 * sizeof(float));
    if (e == cudaSuccess)
        e = ar::launch_refine_patches(dpatch, count, up, drow, dcol, dval, c->num_sms, c->stream);
    if (e == cudaSuccess) e = stage_d2h(c, row, drow, count * 4);
    if (e == cudaSuccess) e = stage_d2h(c, col, dcol, count * 4);
    if (e == cudaSuccess) e = stage_d2h(c, value, dval, count * 4);
    if (e != cudaSuccess) return cuda_fail(c, e, "ar_refine_patches");
    return AR_OK;
}

int ar_prepare(ar_ctx* c, const ar_pair* raw, const ar_prepare_opts* opts, ar_pair** out) {
    if (!c || !raw || !opts || !out) return fail(c, AR_ERR_ARG, "null argument");
    *out = nullptr;
    if (raw->ctx != c) return fail(c, AR_ERR_ARG, "the pair belongs to another context");
    if (opts->preprocess < AR_PRE_NONE || opts->preprocess > AR_PRE_WALLIS)
        return fail(c, AR_ERR_ARG, "unknown preprocess method");
    if (opts->quantize != AR_QUANT_NONE && opts->quantize != AR_QUANT_UINT8)
        return fail(c, AR_ERR_ARG, "unknown quantize method");
    if (opts->preprocess != AR_PRE_NONE) {
        if (opts->width < 3 || (opts->width & 1) == 0)
            return fail(c, AR_ERR_ARG, "filter `width` must be odd and >= 3");
        if (opts->width > ar::max_filter_width())
            return fail(c, AR_ERR_UNSUPPORTED, "filter `width` above the supported maximum");
        if (opts->preprocess == AR_PRE_WALLIS && !(opts->min_std >= 0.0))
            return fail(c, AR_ERR_ARG, "`min_std` must be >= 0");
    }
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    const int64_t n = raw->nrows * raw->ncols;
    const int odt = opts->quantize == AR_QUANT_UINT8 ? AR_U8
                    : (opts->preprocess != AR_PRE_NONE ? AR_F32 : raw->dtype);
    const size_t oes = elem_size(odt);
    ar_pair* p = new ar_pair();
    p->ctx = c;
    p->dtype = odt;
    p->nrows = raw->nrows;
    p->ncols = raw->ncols;
    if (c->scratch.done) cudaStreamWaitEvent(c->stream, c->scratch.done, 0);
    cudaError_t e = dalloc(c, &p->ref, n * oes);
    if (e == cudaSuccess) e = dalloc(c, &p->sec, n * oes);
    if (e == cudaSuccess) e = dalloc(c, &p->valid, 3 * n);
    if (e == cudaSuccess) {
        p->ref_valid = p->valid + n;
        p->sec_valid = p->valid + 2 * n;
    }
    const bool need_f = opts->preprocess != AR_PRE_NONE && opts->quantize == AR_QUANT_UINT8;
    const bool need_m = opts->preprocess == AR_PRE_WALLIS;
    const size_t scratch = (need_f ? n * 4 : 0) + (need_m ? n * 4 : 0) + ar::quant_stats_bytes() + 256;
    unsigned char* tmp = nullptr;
    if (e == cudaSuccess) e = dalloc(c, &tmp, scratch);
    for (int side = 0; side < 2 && e == cudaSuccess; ++side) {
        ar::PrepareJob J{};
        J.dtype = raw->dtype;
        J.img = side == 0 ? raw->ref : raw->sec;
        J.mask = side == 0 ? raw->ref_valid : raw->sec_valid;
        J.nrows = raw->nrows;
        J.ncols = raw->ncols;
        J.preprocess = opts->preprocess;
        J.width = opts->width;
        J.min_std = opts->min_std;
        J.quantize = opts->quantize;
        J.out = side == 0 ? p->ref : p->sec;
        J.vout = side == 0 ? p->ref_valid : p->sec_valid;
        size_t off = 0;
        J.ftmp = need_f ? reinterpret_cast<float*>(tmp + off) : nullptr;
        off += need_f ? n * 4 : 0;
        J.mtmp = need_m ? reinterpret_cast<float*>(tmp + off) : nullptr;
        off += need_m ? n * 4 : 0;
        J.stats = reinterpret_cast<ar::QuantStats*>(tmp + ((off + 255) & ~size_t(255)));
        e = ar::launch_prepare(J, c->stream, &c->scratch.timer.launches);
    }
    if (e == cudaSuccess) {
        const int threads = 256;
        k_and_masks<<<static_cast<unsigned>((n + threads - 1) / threads), threads, 0, c->stream>>>(
            p->ref_valid, p->sec_valid, p->valid, n);
        e = cudaGetLastError();
    }
    dfree(c, tmp);
    if (e == cudaSuccess) e = pair_mark_ready(c, p);
    if (e != cudaSuccess) {
        pair_free(p);
        delete p;
        return cuda_fail(c, e, "ar_prepare");
    }
    *out = p;
    return AR_OK;
}

int ar_pair_download(ar_ctx* c, const ar_pair* p, void* ref, void* sec, uint8_t* ref_valid,
                     uint8_t* sec_valid) {
    if (!c || !p) return fail(c, AR_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    const int64_t n = p->nrows * p->ncols;
    const size_t es = elem_size(p->dtype);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess && ref) e = stage_d2h(c, ref, p->ref, n * es);
    if (e == cudaSuccess && sec) e = stage_d2h(c, sec, p->sec, n * es);
    if (e == cudaSuccess && ref_valid) e = stage_d2h(c, ref_valid, p->ref_valid, n);
    if (e == cudaSuccess && sec_valid) e = stage_d2h(c, sec_valid, p->sec_valid, n);
    return e == cudaSuccess ? AR_OK : cuda_fail(c, e, "ar_pair_download");
}

}  // extern "C"

namespace {

int check_multichip_args(ar_ctx* c, const ar_pair* p, const ar_points* grid, int64_t gr,
                         int64_t gc, const ar_multichip_params* prm) {
    if (!c || !p || !grid || !prm) return fail(c, AR_ERR_ARG, "null argument");
    if (p->ctx != c) return fail(c, AR_ERR_ARG, "the pair belongs to another context");
    if (gr < 0 || gc < 0 || grid->n != gr * gc)
        return fail(c, AR_ERR_SIZE, "grid extents do not match the point count");
    if (grid->n > 0 && (!grid->x || !grid->y || !grid->radius_x || !grid->radius_y ||
                        !grid->dx_prior || !grid->dy_prior))
        return fail(c, AR_ERR_ARG, "null grid field");
    if (!is_pow2(prm->upsampling) || prm->upsampling > 128)
        return fail(c, AR_ERR_ARG, "`upsampling` must be 1 or a power of 2 up to 128");
    if (prm->measure != AR_ZNCC && prm->measure != AR_NCC) return fail(c, AR_ERR_ARG, "unknown measure");
    if (prm->chip_size_base <= 0 || prm->chip_size_max < prm->chip_size_base || prm->coarse_stride <= 0)
        return fail(c, AR_ERR_ARG, "invalid chip-size levels or coarse stride");
    if (prm->rotation_count != 0) {
        ar::Rotation rot;
        std::string err;
        if (!ar::make_rotation(prm->rotation_angles, prm->rotation_count, &rot, &err))
            return fail(c, AR_ERR_ARG, err);
    }
    if (prm->level_measure_count < 0 || prm->level_measure_count > 8)
        return fail(c, AR_ERR_ARG, "level_measure_count must be in [0, 8]");
    int levels = 0;
    for (int64_t cs = prm->chip_size_base; cs <= prm->chip_size_max; cs *= 2)
        if (cs >= prm->chip_size_min) ++levels;
    if (prm->level_measure_count > levels)
        return fail(c, AR_ERR_ARG, "more per-level measures than chip-size levels");
    for (int i = 0; i < prm->level_measure_count; ++i)
        if (prm->level_measures[i] != AR_ZNCC && prm->level_measures[i] != AR_NCC)
            return fail(c, AR_ERR_ARG, "unknown per-level measure");
    return AR_OK;
}

// The search over a grid whose fields and outputs are device arrays; the caller holds the
// context lock. Returns once the search has completed on `s`.
int multichip_run(ar_ctx* c, const ar_pair* p, const double* gx, const double* gy,
                  const int64_t* grx, const int64_t* gry, const double* gdx0, const double* gdy0,
                  int64_t gr, int64_t gc, const ar_multichip_params* prm, float* dx, float* dy,
                  float* corr, uint16_t* chip, uint8_t* interp, cudaStream_t s) {
    const cudaError_t ew = pair_wait(c, p, s);
    if (ew != cudaSuccess) return cuda_fail(c, ew, "ar_multichip: pair");
    // The search's scratch is kept by the context and grows from its pool in stream order on
    // `s` (no device-wide synchronisation, so the request loop's slots never stall one
    // another). Every call ends with its stream synchronised, so the scratch is idle when the
    // next call (on any stream) takes it. Kept rather than taken and returned per call: a
    // block of this size returned to the pool between calls made later allocations slower.
    const size_t ab = ar::multichip_arena_bytes(gr, gc);
    if (c->arena_bytes < ab) {
        if (c->arena) cudaFreeAsync(c->arena, s);
        c->arena = nullptr;
        c->arena_bytes = 0;
        cudaError_t ea = cudaMallocFromPoolAsync(&c->arena, ab, c->pool, s);
        if (ea != cudaSuccess) return cuda_fail(c, ea, "ar_multichip: scratch");
        c->arena_bytes = ab;
    }
    void* arena = c->arena;
    ar::MultichipJob J{};
    J.dtype = p->dtype;
    J.ref = p->ref;
    J.sec = p->sec;
    J.valid = p->valid;
    J.nrows = p->nrows;
    J.ncols = p->ncols;
    J.gx = gx;
    J.gy = gy;
    J.grx = grx;
    J.gry = gry;
    J.gdx0 = gdx0;
    J.gdy0 = gdy0;
    J.gr = gr;
    J.gc = gc;
    J.dx = dx;
    J.dy = dy;
    J.corr = corr;
    J.chip = chip;
    J.interp = interp;
    ar::MultichipParams& P = J.P;
    P.chip_base = prm->chip_size_base;
    P.chip_min = prm->chip_size_min;
    P.chip_max = prm->chip_size_max;
    P.aspect = prm->chip_aspect;
    P.min_radius = prm->min_search_radius;
    P.stride = prm->coarse_stride;
    P.buffer = prm->coarse_buffer;
    P.min_frac = prm->min_coarse_valid_fraction;
    P.up = prm->upsampling;
    P.measure = prm->measure;
    P.outliers = prm->outliers;
    P.gwindow = prm->outlier_window;
    P.giterations = prm->outlier_iterations;
    P.gfrac = prm->min_agree_fraction;
    P.gtol = prm->agree_tolerance;
    P.gmad = prm->mad_scale;
    P.fill_window = prm->fill_window;
    if (prm->rotation_count != 0)
        ar::make_rotation(prm->rotation_angles, prm->rotation_count, &P.rot, nullptr);
    P.n_level_measures = prm->level_measure_count;
    for (int i = 0; i < 8; ++i)
        P.level_measures[i] = i < prm->level_measure_count ? prm->level_measures[i] : prm->measure;
    J.arena = arena;
    J.arena_bytes = ab;
    std::string err;
    cudaError_t e = ar::run_multichip(J, c->scratch, c->num_sms, s, &err);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return err.empty() ? cuda_fail(c, e, "ar_multichip") : fail(c, AR_ERR_UNSUPPORTED, err);
    int st = 0;
    e = ar::read_status(c->scratch, s, &st);
    if (e != cudaSuccess) return cuda_fail(c, e, "ar_multichip: status");
    if (st) return fail(c, AR_ERR_TIMEOUT, "ar_multichip: a device wait ran out; results incomplete");
    return AR_OK;
}

}  // namespace

extern "C" {

int ar_multichip(ar_ctx* c, const ar_pair* p, const ar_points* grid, int64_t gr, int64_t gc,
                 const ar_multichip_params* prm, float* dx, float* dy, float* corr,
                 uint16_t* chip, uint8_t* interp) {
    int rc = check_multichip_args(c, p, grid, gr, gc, prm);
    if (rc != AR_OK) return rc;
    const int64_t n = grid->n;
    if (n == 0) return AR_OK;
    if (!dx || !dy || !corr || !chip || !interp) return fail(c, AR_ERR_ARG, "null output");
    for (int64_t k = 0; k < n; ++k)
        if (!std::isfinite(grid->x[k]) || !std::isfinite(grid->y[k]) ||
            !std::isfinite(grid->dx_prior[k]) || !std::isfinite(grid->dy_prior[k]))
            return fail(c, AR_ERR_ARG, "grid coordinates and priors must be finite");
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    // Device copies of the six grid fields and the five outputs.
    const size_t need = static_cast<size_t>(n) * (6 * 8 + 3 * 4 + 2 + 1) + 16 * 256;
    cudaError_t e = ensure_dbuf(c, need);
    if (e != cudaSuccess) return cuda_fail(c, e, "ar_multichip: device buffers");
    unsigned char* base = static_cast<unsigned char*>(c->dbuf);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        off = (off + 255) & ~size_t(255);
        unsigned char* q = base + off;
        off += bytes;
        return q;
    };
    double* gx = reinterpret_cast<double*>(take(n * 8));
    double* gy = reinterpret_cast<double*>(take(n * 8));
    int64_t* grx = reinterpret_cast<int64_t*>(take(n * 8));
    int64_t* gry = reinterpret_cast<int64_t*>(take(n * 8));
    double* gdx0 = reinterpret_cast<double*>(take(n * 8));
    double* gdy0 = reinterpret_cast<double*>(take(n * 8));
    float* ddx = reinterpret_cast<float*>(take(n * 4));
    float* ddy = reinterpret_cast<float*>(take(n * 4));
    float* dcorr = reinterpret_cast<float*>(take(n * 4));
    uint16_t* dchip = reinterpret_cast<uint16_t*>(take(n * 2));
    uint8_t* dint = take(n);
    const void* srcs[6] = {grid->x, grid->y, grid->radius_x, grid->radius_y, grid->dx_prior, grid->dy_prior};
    void* dsts[6] = {gx, gy, grx, gry, gdx0, gdy0};
    for (int f = 0; f < 6 && e == cudaSuccess; ++f) e = stage_h2d(c, dsts[f], srcs[f], n * 8);
    if (e != cudaSuccess) return cuda_fail(c, e, "ar_multichip: upload grid");
    rc = multichip_run(c, p, gx, gy, grx, gry, gdx0, gdy0, gr, gc, prm, ddx, ddy, dcorr, dchip,
                       dint, c->stream);
    if (rc != AR_OK) return rc;
    e = stage_d2h(c, dx, ddx, n * 4);
    if (e == cudaSuccess) e = stage_d2h(c, dy, ddy, n * 4);
    if (e == cudaSuccess) e = stage_d2h(c, corr, dcorr, n * 4);
    if (e == cudaSuccess) e = stage_d2h(c, chip, dchip, n * 2);
    if (e == cudaSuccess) e = stage_d2h(c, interp, dint, n);
    if (e != cudaSuccess) return cuda_fail(c, e, "ar_multichip: download");
    return AR_OK;
}

int ar_multichip_device(ar_ctx* c, const ar_pair* p, const ar_points* grid, int64_t gr,
                        int64_t gc, const ar_multichip_params* prm, float* dx, float* dy,
                        float* corr, uint16_t* chip, uint8_t* interp, void* stream) {
    int rc = check_multichip_args(c, p, grid, gr, gc, prm);
    if (rc != AR_OK) return rc;
    if (grid->n == 0) return AR_OK;
    if (!dx || !dy || !corr || !chip || !interp) return fail(c, AR_ERR_ARG, "null output");
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    return multichip_run(c, p, grid->x, grid->y, grid->radius_x, grid->radius_y, grid->dx_prior,
                         grid->dy_prior, gr, gc, prm, dx, dy, corr, chip, interp, s);
}

int ar_tc_selftest(ar_ctx* c, const uint8_t* a_img, int a_bytes, const uint8_t* b_img,
                   int b_bytes, const int* params, int32_t* d_out) {
    if (!c || !a_img || !b_img || !params || !d_out) return fail(c, AR_ERR_ARG, "null argument");
    if (a_bytes <= 0 || b_bytes <= 0 || a_bytes > 96 * 1024 || b_bytes > 96 * 1024)
        return fail(c, AR_ERR_SIZE, "operand images must be 1..96 KiB");
    const int N = params[9], nk = params[10], dstep = params[11];
    // params[12]: 0 reads the accumulator lane by lane (32x32b), 1 with the 16x256b pattern.
    if (N < 8 || N > 256 || nk < 1 || nk > 64 || dstep < 0 || dstep > 512)
        return fail(c, AR_ERR_ARG, "invalid N, nk or dstep");
    const int dcols = N + (nk - 1) * dstep;
    if (dcols > 512) return fail(c, AR_ERR_ARG, "the accumulator columns exceed Tensor Memory");
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    unsigned char *da = nullptr, *db = nullptr, *dd = nullptr;
    const size_t dbytes = static_cast<size_t>(128) * dcols * 4 + 16;
    cudaError_t e = dalloc(c, &da, a_bytes);
    if (e == cudaSuccess) e = dalloc(c, &db, b_bytes);
    if (e == cudaSuccess) e = dalloc(c, &dd, dbytes);
    if (e == cudaSuccess) e = cudaMemcpyAsync(da, a_img, a_bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(db, b_img, b_bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(dd, 0, dbytes, c->stream);
    int* status = reinterpret_cast<int*>(dd + static_cast<size_t>(128) * dcols * 4);
    std::string err;
    if (e == cudaSuccess)
        e = ar::tc_probe(da, a_bytes, db, b_bytes, params, reinterpret_cast<int32_t*>(dd), status,
                         c->stream, &err);
    int hstatus = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_out, dd, static_cast<size_t>(128) * dcols * 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&hstatus, status, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    dfree(c, da);
    dfree(c, db);
    dfree(c, dd);
    if (e != cudaSuccess)
        return err.empty() ? cuda_fail(c, e, "ar_tc_selftest") : fail(c, AR_ERR_ARG, err);
    if (hstatus != 0) return fail(c, AR_ERR_TIMEOUT, "the tensor-core product did not complete in time");
    return AR_OK;
}

int ar_ctx_set_option(ar_ctx* c, int option, int value) {
    if (!c) return AR_ERR_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    switch (option) {
        case AR_OPT_TENSOR_CORES: c->scratch.tensor_cores = value != 0; return AR_OK;
        case AR_OPT_AUTOTUNE: c->scratch.autotune = value != 0; return AR_OK;
        case AR_OPT_SHAPE_BINS: c->scratch.shape_bins = value != 0; return AR_OK;
        case AR_OPT_UINT8_KERNEL:
            if (value < -1 || value > 2) return fail(c, AR_ERR_ARG, "the UInt8 kernel must be -1, 0, 1 or 2");
            c->scratch.uint8_kernel = value;
            return AR_OK;
        case AR_OPT_SPLIT_BF16:
            if (value < 0 || value > 2) return fail(c, AR_ERR_ARG, "split-BF16 mode must be 0, 1 or 2");
            c->scratch.split_bf16 = value;
            return AR_OK;
        case AR_OPT_SERVE_SLOTS:
        case AR_OPT_SERVE_MEMORY_MB: {
            std::lock_guard<std::mutex> sk(c->serve_mu);
            if (c->serve) return fail(c, AR_ERR_ARG, "the request loop has already started");
            if (option == AR_OPT_SERVE_SLOTS) {
                if (value < 1 || value > 64) return fail(c, AR_ERR_ARG, "slots must be in 1..64");
                c->serve_slots = value;
            } else {
                if (value < 0) return fail(c, AR_ERR_ARG, "the memory budget must be >= 0");
                c->serve_budget = static_cast<size_t>(value) << 20;
            }
            return AR_OK;
        }
        default: return fail(c, AR_ERR_ARG, "unknown option");
    }
}

int ar_submit(ar_ctx* c, const ar_request* req, ar_ticket* ticket) {
    if (!c || !req || !ticket) return fail(c, AR_ERR_ARG, "null argument");
    ar::ServeEngine* E;
    {
        std::lock_guard<std::mutex> lk(c->serve_mu);
        if (!c->serve) {
            std::string err;
            c->serve = ar::serve_create(c->device, c->serve_slots, c->serve_budget, &err);
            if (!c->serve) return fail(c, AR_ERR_CUDA, "ar_submit: " + err);
        }
        E = c->serve;
    }
    std::string err;
    int64_t t = 0;
    const int rc = ar::serve_submit(E, req, &t, &err);
    if (rc != AR_OK) return fail(c, rc, "ar_submit: " + err);
    *ticket = t;
    return AR_OK;
}

namespace {
ar::ServeEngine* engine_of(ar_ctx* c) {
    std::lock_guard<std::mutex> lk(c->serve_mu);
    return c->serve;
}
}  // namespace

int ar_poll(ar_ctx* c, ar_ticket ticket, int* done) {
    if (!c || !done) return fail(c, AR_ERR_ARG, "null argument");
    ar::ServeEngine* E = engine_of(c);
    if (!E) return fail(c, AR_ERR_ARG, "no request has been submitted");
    std::string err;
    const int rc = ar::serve_poll(E, ticket, done, &err);
    return rc == AR_OK ? AR_OK : fail(c, rc, err);
}

int ar_wait(ar_ctx* c, ar_ticket ticket, int timeout_ms) {
    if (!c) return AR_ERR_ARG;
    ar::ServeEngine* E = engine_of(c);
    if (!E) return fail(c, AR_ERR_ARG, "no request has been submitted");
    std::string err;
    const int rc = ar::serve_wait(E, ticket, timeout_ms, &err);
    return rc == AR_OK ? AR_OK : fail(c, rc, err);
}

int ar_request_times(ar_ctx* c, ar_ticket ticket, double* queued_ms, double* run_ms) {
    if (!c) return AR_ERR_ARG;
    ar::ServeEngine* E = engine_of(c);
    if (!E) return fail(c, AR_ERR_ARG, "no request has been submitted");
    const int rc = ar::serve_times(E, ticket, queued_ms, run_ms);
    return rc == AR_OK ? AR_OK : fail(c, rc, "unknown or pending ticket");
}

int ar_release(ar_ctx* c, ar_ticket ticket) {
    if (!c) return AR_ERR_ARG;
    ar::ServeEngine* E = engine_of(c);
    if (!E) return fail(c, AR_ERR_ARG, "no request has been submitted");
    std::string err;
    const int rc = ar::serve_release(E, ticket, &err);
    return rc == AR_OK ? AR_OK : fail(c, rc, err);
}

int ar_ctx_stream(ar_ctx* c, void** stream) {
    if (!c || !stream) return AR_ERR_ARG;
    *stream = c->stream;
    return AR_OK;
}

int ar_ctx_set_timing(ar_ctx* c, int enable) {
    if (!c) return AR_ERR_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    ar::KernelTimer& T = c->scratch.timer;
    if (enable && !T.flops) {
        cudaError_t e = cudaMalloc(&T.flops, sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMemsetAsync(T.flops, 0, sizeof(unsigned long long), c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "ar_ctx_set_timing");
    }
    T.enabled = enable != 0;
    return AR_OK;
}

int ar_kernel_times(ar_ctx* c, double* corr_ms, double* refine_ms, int64_t* tracks,
                    int64_t* launches, double* corr_flops) {
    if (!c) return AR_ERR_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    DeviceGuard g(c->device);
    ar::KernelTimer& T = c->scratch.timer;
    double sc = 0.0, sr = 0.0;
    cudaError_t e = cudaSuccess;
    for (auto& r : T.recs) {
        float a = 0.0f, b = 0.0f;
        if (e == cudaSuccess) e = cudaEventSynchronize(r[2]);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&a, r[0], r[1]);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&b, r[1], r[2]);
        sc += a;
        sr += b;
        for (auto ev : r) T.pool.push_back(ev);
    }
    if (tracks) *tracks = static_cast<int64_t>(T.recs.size());
    if (launches) *launches = T.launches;
    unsigned long long fl = 0;
    if (T.flops) {
        if (e == cudaSuccess) e = cudaMemcpy(&fl, T.flops, sizeof(fl), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemset(T.flops, 0, sizeof(fl));
    }
    if (corr_flops) *corr_flops = static_cast<double>(fl);
    T.recs.clear();
    T.launches = 0;
    if (corr_ms) *corr_ms = sc;
    if (refine_ms) *refine_ms = sr;
    return e == cudaSuccess ? AR_OK : cuda_fail(c, e, "ar_kernel_times");
}

int ar_ctx_tuned(ar_ctx* c, int32_t* out, int64_t cap, int64_t* count) {
    if (!c || !count || cap < 0 || (cap > 0 && !out)) return AR_ERR_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    int64_t n = 0;
    for (const auto& kv : c->scratch.tuned) {
        if (n < cap) {
            int32_t* o = out + 5 * n;
            o[0] = static_cast<int32_t>((kv.first >> 48) & 0xFFFF);
            o[1] = static_cast<int32_t>((kv.first >> 32) & 0xFFFF);
            o[2] = static_cast<int32_t>((kv.first >> 16) & 0xFFFF);
            o[3] = static_cast<int32_t>(kv.first & 0xFFFF);
            o[4] = kv.second;
        }
        ++n;
    }
    *count = n;
    return AR_OK;
}

int ar_synchronize(ar_ctx* c) {
    if (!c) return AR_ERR_ARG;
    DeviceGuard g(c->device);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? AR_OK : cuda_fail(c, e, "ar_synchronize");
}

}  // extern "C"
