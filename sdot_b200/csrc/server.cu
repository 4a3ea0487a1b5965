// Serving loop: semi-discrete OT solves of uneven sizes, continuously batched
// (see the sdot_server_* block of include/sdot_gpu.h).
//
// A server owns `slots` workers.  Each worker has its own contexts (one per
// dimension, so grids, weights, Hessian rows and solver buffers stay resident
// and are reused by the next request of that dimension) and therefore its own
// CUDA stream.  Requests are admitted in arrival order as soon as a worker is
// free and the estimated device memory of the requests in flight stays under
// the budget; while one request waits on its stream (the Newton loop reads a
// few scalars back per iteration), the others keep the GPU busy, so the work
// of requests in flight overlaps on the device.  slots = 1 is the sequential
// baseline: one plain solve after the other.
//
// Each worker holds a high- and a low-priority CUDA stream; requests of at
// least HIGH_PRIORITY_BYTES (the long solves that set the tail latency) run
// on the high one, so that the GPU's block scheduler serves their kernels
// first and they keep close to their solo speed while the smaller requests
// fill the gaps.
#include "../../include/sdot_gpu.h"

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

struct Request {
    int dim = 2;
    int64_t n = 0;
    std::vector<double> pos, w, target;
    double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
    int64_t bytes = 0;
    // results
    int status = SDOT_PENDING;
    std::vector<double> weights;
    sdot_request_report report{};
    std::string error;
};

// Device memory a request needs beyond its worker's fixed buffers: Diracs,
// tree, cell outputs, Hessian rows (ELL) and solver vectors, per Dirac.
int64_t request_bytes(int dim, int64_t n) { return n * (dim == 3 ? 1400 : 800) + (1 << 20); }
constexpr int64_t HIGH_PRIORITY_BYTES = int64_t(64) << 20;  // 3D from ~47k Diracs, 2D from ~83k

}  // namespace

struct sdot_server {
    sdot_server_opts opts{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<int64_t> queue;  // admitted in this order
    std::vector<std::unique_ptr<Request>> reqs;
    int64_t in_flight_bytes = 0;
    int running = 0;
    bool stopping = false;
    std::vector<std::thread> workers;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }

    void worker_main() {
        sdot_ctx *ctx[2] = {nullptr, nullptr};
        sdot_options o{};
        o.max_diracs_per_cell = 11;
        o.stream = nullptr;
        o.device = opts.device;
        cudaStream_t hi = nullptr, lo = nullptr;
        {
            int least = 0, greatest = 0;
            if (opts.device >= 0) cudaSetDevice(opts.device);
            if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
                cudaStreamCreateWithPriority(&hi, cudaStreamNonBlocking, greatest) != cudaSuccess ||
                cudaStreamCreateWithPriority(&lo, cudaStreamNonBlocking, least) != cudaSuccess) {
                cudaGetLastError();
                if (hi) cudaStreamDestroy(hi);
                hi = lo = nullptr;  // the contexts' own streams then
            }
        }
        while (true) {
            int64_t id = -1;
            Request *r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                // the head of the queue starts when its memory fits (or when
                // nothing else runs: a request larger than the budget still
                // runs, alone)
                cv_work.wait(lk, [&] {
                    if (stopping) return true;
                    if (queue.empty()) return false;
                    const Request &h = *reqs[queue.front()];
                    return running == 0 || in_flight_bytes + h.bytes <= opts.hbm_budget_bytes;
                });
                if (stopping && queue.empty()) break;
                if (queue.empty()) continue;
                id = queue.front();
                queue.pop_front();
                r = reqs[id].get();
                in_flight_bytes += r->bytes;
                ++running;
                r->report.start_ms = now_ms();
            }
            const int k = r->dim == 3 ? 1 : 0;
            int st = SDOT_OK;
            if (!ctx[k]) ctx[k] = sdot_create(r->dim, SDOT_FP64, &o);
            if (!ctx[k]) {
                st = SDOT_CUDA_ERROR;
                r->error = "sdot_create failed";
            }
            sdot_newton_report rep{};
            if (st == SDOT_OK && hi) st = sdot_set_stream(ctx[k], r->bytes >= HIGH_PRIORITY_BYTES ? hi : lo);
            if (st == SDOT_OK) st = sdot_clear_domain(ctx[k]);
            if (st == SDOT_OK) st = sdot_add_box_shape(ctx[k], r->lo, r->hi, 1.0);
            if (st == SDOT_OK) st = sdot_set_diracs(ctx[k], r->pos.data(), r->w.data(), r->n, SDOT_HOST);
            if (st == SDOT_OK) st = sdot_solve(ctx[k], r->target.data(), SDOT_HOST, &opts.newton, &rep);
            r->weights.resize(size_t(r->n));
            const int st2 = ctx[k] ? sdot_get_weights(ctx[k], r->weights.data(), SDOT_HOST) : SDOT_CUDA_ERROR;
            if (st == SDOT_OK) st = st2;
            if (st != SDOT_OK && ctx[k] && r->error.empty()) r->error = sdot_last_error(ctx[k]);
            {
                std::lock_guard<std::mutex> lk(mu);
                r->report.end_ms = now_ms();
                r->report.status = st;
                r->report.iterations = rep.iterations;
                r->report.max_rel_mass_error = rep.max_rel_mass_error;
                r->status = st;
                in_flight_bytes -= r->bytes;
                --running;
            }
            cv_work.notify_all();
            cv_done.notify_all();
        }
        for (sdot_ctx *c : ctx)
            if (c) sdot_destroy(c);
        if (hi) cudaStreamDestroy(hi);
        if (lo) cudaStreamDestroy(lo);
    }
};

extern "C" {

sdot_server *sdot_server_create(const sdot_server_opts *opts) {
    if (!opts || opts->slots < 1 || opts->slots > 64 || opts->hbm_budget_bytes <= 0) return nullptr;
    sdot_server *s = nullptr;
    try {
        s = new sdot_server();
        s->opts = *opts;
        for (int i = 0; i < opts->slots; ++i) s->workers.emplace_back([s] { s->worker_main(); });
    } catch (...) {
        if (s) {
            {
                std::lock_guard<std::mutex> lk(s->mu);
                s->stopping = true;
            }
            s->cv_work.notify_all();
            for (auto &t : s->workers) t.join();
            delete s;
        }
        return nullptr;
    }
    return s;
}

int64_t sdot_server_submit(sdot_server *srv, int dim, int64_t n, const double *positions, const double *weights,
                           const double *target, const double *box_lo, const double *box_hi) {
    if (!srv || (dim != 2 && dim != 3) || n <= 0 || !positions || !target) return -SDOT_BAD_ARG;
    try {
        auto r = std::make_unique<Request>();
        r->dim = dim;
        r->n = n;
        r->pos.assign(positions, positions + size_t(dim) * n);
        if (weights)
            r->w.assign(weights, weights + n);
        else
            r->w.assign(size_t(n), 0.0);
        r->target.assign(target, target + n);
        for (int d = 0; d < dim; ++d) {
            r->lo[d] = box_lo ? box_lo[d] : 0.0;
            r->hi[d] = box_hi ? box_hi[d] : 1.0;
        }
        r->bytes = request_bytes(dim, n);
        std::lock_guard<std::mutex> lk(srv->mu);
        r->report.submit_ms = srv->now_ms();
        r->report.status = SDOT_PENDING;
        const int64_t id = int64_t(srv->reqs.size());
        srv->reqs.push_back(std::move(r));
        srv->queue.push_back(id);
        srv->cv_work.notify_one();
        return id;
    } catch (...) {
        return -SDOT_OOM;
    }
}

int sdot_server_poll(sdot_server *srv, int64_t id, double *weights_out, sdot_request_report *report) {
    if (!srv) return SDOT_BAD_ARG;
    std::lock_guard<std::mutex> lk(srv->mu);
    if (id < 0 || id >= int64_t(srv->reqs.size())) return SDOT_BAD_ARG;
    const Request &r = *srv->reqs[id];
    if (report) *report = r.report;
    if (r.status == SDOT_PENDING) return SDOT_PENDING;
    if (weights_out && !r.weights.empty()) std::memcpy(weights_out, r.weights.data(), r.weights.size() * sizeof(double));
    return r.status;
}

int sdot_server_drain(sdot_server *srv) {
    if (!srv) return SDOT_BAD_ARG;
    std::unique_lock<std::mutex> lk(srv->mu);
    srv->cv_done.wait(lk, [&] { return srv->queue.empty() && srv->running == 0; });
    return SDOT_OK;
}

void sdot_server_destroy(sdot_server *srv) {
    if (!srv) return;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stopping = true;
    }
    srv->cv_work.notify_all();
    for (auto &t : srv->workers) t.join();
    delete srv;
}

}  // extern "C"
