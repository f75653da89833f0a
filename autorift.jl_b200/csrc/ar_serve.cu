// The request loop of a context: continuous batching of whole autorift() requests.
//
// A request is a pair of host images plus a grid and the parameters of the default pipeline
// (the reference's `autorift(image1, image2; ...)`, src/api.jl:210-274: prepare both images,
// then the multi-chip-size search, src/multichip.jl:106-422). Requests queue in submission
// order; each of the engine's slots -- a context of its own (stream, scratch, memory pool)
// driven by one host thread -- takes the next request once the device memory the admitted
// requests may hold (their footprint) leaves room for it. Requests that arrive while others run
// are admitted as slots and memory free up, and their kernels overlap on the device: one
// request's host-side steps (uploads, the per-level counter reads of the search) leave the
// device to the others. Results are bit-identical to running each request alone: every kernel
// is deterministic and a slot's scratch belongs to it.

#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ar_internal.cuh"

namespace ar {

namespace {

using Clock = std::chrono::steady_clock;

constexpr int kPending = -1;

struct Job {
    int64_t ticket = 0;
    ar_request req{};
    std::vector<double> angles;  // the request's rotation angles, copied at submission
    size_t footprint = 0;
    int status = kPending;
    std::string err;
    Clock::time_point t_submit, t_start, t_end;
};

size_t elem_bytes(int dtype) {
    switch (dtype) {
        case AR_U8: return 1;
        case AR_U16: return 2;
        case AR_I16: return 2;
        case AR_F32: return 4;
        default: return 0;
    }
}

}  // namespace

struct ServeEngine {
    int device = 0;
    std::vector<ar_ctx*> slots;
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Job>> queue;
    std::unordered_map<int64_t, std::shared_ptr<Job>> jobs;
    size_t budget = 0, in_use = 0;
    int running = 0;
    int64_t next = 1;
    bool stop = false;
};

namespace {

// Device bytes a request can hold at once: the raw pair, the prepared pair, the filter scratch,
// the grid with its outputs, the search's scratch and the track queue.
size_t footprint(const ar_request& r) {
    const size_t n = static_cast<size_t>(r.nrows) * static_cast<size_t>(r.ncols);
    const size_t es = elem_bytes(r.dtype);
    const size_t oes = r.prepare.quantize == AR_QUANT_UINT8 ? 1 : (r.prepare.preprocess ? 4 : es);
    const size_t g = static_cast<size_t>(r.grid_rows) * static_cast<size_t>(r.grid_cols);
    size_t b = n * (2 * es + 3) + n * (2 * oes + 3);
    b += n * 4 * (r.prepare.preprocess ? 1 : 0) + n * 4 * (r.prepare.preprocess == AR_PRE_WALLIS ? 1 : 0);
    b += g * (6 * 8 + 15) + multichip_arena_bytes(r.grid_rows, r.grid_cols) + g * 128;
    return b + (16u << 20);
}

std::string slot_error(ar_ctx* c) {
    char buf[512];
    ar_last_error(c, buf, sizeof(buf));
    return std::string(buf);
}

int run_job(ar_ctx* c, Job& j) {
    const ar_request& r = j.req;
    ar_pair* raw = nullptr;
    ar_pair* prep = nullptr;
    int rc = ar_pair_upload(c, r.reference, r.secondary, r.reference_valid, r.secondary_valid,
                            r.nrows, r.ncols, r.dtype, &raw);
    if (rc == AR_OK) rc = ar_prepare(c, raw, &r.prepare, &prep);
    if (raw) ar_pair_destroy(raw);  // free the raw images before the search
    if (rc == AR_OK)
        rc = ar_multichip(c, prep, r.grid, r.grid_rows, r.grid_cols, &r.params, r.dx, r.dy,
                          r.correlation, r.chip_size, r.interpolated);
    if (rc != AR_OK) j.err = slot_error(c);
    if (prep) ar_pair_destroy(prep);
    return rc;
}

void worker(ServeEngine* E, int s) {
    ar_ctx* c = E->slots[s];
    for (;;) {
        std::shared_ptr<Job> job;
        {
            std::unique_lock<std::mutex> lk(E->mu);
            E->cv_work.wait(lk, [&] {
                if (E->queue.empty()) return E->stop;
                const size_t fp = E->queue.front()->footprint;
                return E->running == 0 || E->in_use + fp <= E->budget;
            });
            if (E->queue.empty()) return;  // stopping and drained
            job = E->queue.front();
            E->queue.pop_front();
            E->in_use += job->footprint;
            ++E->running;
            job->t_start = Clock::now();
        }
        const int rc = run_job(c, *job);
        {
            std::lock_guard<std::mutex> lk(E->mu);
            E->in_use -= job->footprint;
            --E->running;
            job->t_end = Clock::now();
            job->status = rc;
        }
        E->cv_done.notify_all();
        E->cv_work.notify_all();
    }
}

}  // namespace

ServeEngine* serve_create(int device, int slots, size_t budget, std::string* err) {
    auto* E = new ServeEngine();
    E->device = device;
    for (int s = 0; s < slots; ++s) {
        ar_ctx* c = nullptr;
        if (ar_ctx_create(device, &c) != AR_OK) {
            if (err) *err = "could not create the serving slots' contexts";
            for (ar_ctx* x : E->slots) ar_ctx_destroy(x);
            delete E;
            return nullptr;
        }
        E->slots.push_back(c);
    }
    if (budget == 0) {
        size_t free_b = 0, total_b = 0;
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        cudaMemGetInfo(&free_b, &total_b);
        cudaSetDevice(prev);
        budget = free_b / 4 * 3;  // three quarters of what is free when serving starts
    }
    E->budget = budget;
    for (int s = 0; s < slots; ++s) E->workers.emplace_back(worker, E, s);
    return E;
}

void serve_destroy(ServeEngine* E) {
    if (!E) return;
    {
        std::lock_guard<std::mutex> lk(E->mu);
        E->stop = true;
    }
    E->cv_work.notify_all();
    for (auto& t : E->workers) t.join();
    for (ar_ctx* c : E->slots) ar_ctx_destroy(c);
    delete E;
}

int serve_submit(ServeEngine* E, const ar_request* r, int64_t* ticket, std::string* err) {
    if (!r->reference || !r->secondary || !r->grid || !r->dx || !r->dy || !r->correlation ||
        !r->chip_size || !r->interpolated) {
        *err = "null image, grid or output pointer";
        return AR_ERR_ARG;
    }
    if (r->nrows <= 0 || r->ncols <= 0) {
        *err = "image extents must be positive";
        return AR_ERR_SIZE;
    }
    if (elem_bytes(r->dtype) == 0) {
        *err = "unsupported element type";
        return AR_ERR_UNSUPPORTED;
    }
    if (r->grid_rows < 0 || r->grid_cols < 0 || r->grid->n != r->grid_rows * r->grid_cols) {
        *err = "grid extents do not match the point count";
        return AR_ERR_SIZE;
    }
    if (r->params.rotation_count != 0) {
        Rotation rot;
        if (!make_rotation(r->params.rotation_angles, r->params.rotation_count, &rot, err))
            return AR_ERR_ARG;
    }
    auto j = std::make_shared<Job>();
    j->req = *r;
    if (r->params.rotation_count != 0) {
        j->angles.assign(r->params.rotation_angles,
                         r->params.rotation_angles + r->params.rotation_count);
        j->req.params.rotation_angles = j->angles.data();
    }
    j->footprint = footprint(*r);
    j->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(E->mu);
        if (E->stop) {
            *err = "the context is shutting down";
            return AR_ERR_ARG;
        }
        j->ticket = E->next++;
        E->jobs[j->ticket] = j;
        E->queue.push_back(j);
    }
    E->cv_work.notify_one();
    *ticket = j->ticket;
    return AR_OK;
}

// Completed: the request's status (its message into `err`).
static int finish(const Job& j, std::string* err) {
    if (j.status != AR_OK) *err = j.err;
    return j.status;
}

int serve_poll(ServeEngine* E, int64_t ticket, int* done, std::string* err) {
    std::lock_guard<std::mutex> lk(E->mu);
    auto it = E->jobs.find(ticket);
    if (it == E->jobs.end()) {
        *err = "unknown ticket (never issued, or released)";
        return AR_ERR_ARG;
    }
    if (it->second->status == kPending) {
        *done = 0;
        return AR_OK;
    }
    *done = 1;
    return finish(*it->second, err);
}

int serve_wait(ServeEngine* E, int64_t ticket, int timeout_ms, std::string* err) {
    std::unique_lock<std::mutex> lk(E->mu);
    auto it = E->jobs.find(ticket);
    if (it == E->jobs.end()) {
        *err = "unknown ticket (never issued, or released)";
        return AR_ERR_ARG;
    }
    std::shared_ptr<Job> j = it->second;
    auto ready = [&] { return j->status != kPending; };
    if (timeout_ms < 0) {
        E->cv_done.wait(lk, ready);
    } else if (!E->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
        *err = "the request has not completed within the timeout";
        return AR_ERR_TIMEOUT;
    }
    return finish(*j, err);
}

int serve_release(ServeEngine* E, int64_t ticket, std::string* err) {
    std::lock_guard<std::mutex> lk(E->mu);
    auto it = E->jobs.find(ticket);
    if (it == E->jobs.end()) {
        *err = "unknown ticket";
        return AR_ERR_ARG;
    }
    if (it->second->status == kPending) {
        *err = "the request has not completed";
        return AR_ERR_ARG;
    }
    E->jobs.erase(it);
    return AR_OK;
}

int serve_times(ServeEngine* E, int64_t ticket, double* queued_ms, double* run_ms) {
    std::lock_guard<std::mutex> lk(E->mu);
    auto it = E->jobs.find(ticket);
    if (it == E->jobs.end() || it->second->status == kPending) return AR_ERR_ARG;
    const Job& j = *it->second;
    using ms = std::chrono::duration<double, std::milli>;
    if (queued_ms) *queued_ms = ms(j.t_start - j.t_submit).count();
    if (run_ms) *run_ms = ms(j.t_end - j.t_start).count();
    return AR_OK;
}

}  // namespace ar
