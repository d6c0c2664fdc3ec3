// Self-join request server: continuous batching of independent self-joins.
//
// Requests are admitted as soon as the server has a free slot and the device
// memory they need (scratch + their resident result) fits in its budget: the
// waiting request with the fewest cells first, so that under load a small
// request does not queue behind large ones for a slot, except that a request
// that has waited kAgeLimitS goes before any other, so none starves.  A
// finished profile stays in device memory until the client collects it, and
// its memory counts against the budget until then.  A request larger than the
// whole budget is rejected at submission.  No counterpart in
// the reference (one join per process there).
//
// FP32 re-anchored form: one scheduler thread runs the admitted requests as
// epochs (mp_serve.h).  Each epoch is one persistent launch of the FP32 tile
// kernel over a bounded slice of tiles (about kEpochCells cells) drawn from
// every admitted request: each request first gets a minimum share, then the
// rest goes to the requests with the least work left, so a small request
// that arrives while a large one runs is finished within an epoch or two.
// New requests are prepared on the same stream between epochs; two epochs are
// kept in flight so the GPU never waits for the scheduler.  Device memory
// comes from a server-owned stream-ordered pool, so no allocation or release
// waits for the device.
// FP64 and guarded FP32 forms: worker threads, each running whole
// mp_selfjoin calls on its own stream and context, with each call's scratch
// and result taken from the same pool (the scratch lent to the context for
// the call), so the budget counts all of it and nothing waits on cudaFree.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <set>
#include <thread>
#include <unordered_map>
#include <vector>

#include "mp_serve.h"
#include "mpgpu.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t id = 0;
    std::vector<double> series;
    int64_t m = 0, PL = 0;
    double cells = 0.0;    // cells of the join (the admission order)
    size_t need = 0;       // device bytes while running: scratch + resident result
    size_t accounted = 0;  // bytes of this request currently counted in in_use
    Clock::time_point submitted, started, finished;
    int status = -1;  // -1 pending, >= 0 final status
    double* d_d2 = nullptr;
    int64_t* d_idx = nullptr;
    bool collected = false;
    mpgpu::ServeJob job;  // epoch mode
};

}  // namespace

struct mp_server {
    int device = 0;
    size_t budget = 0;
    int precision = MP_PREC_FP32_REANCHOR;
    int64_t reanchor_k = 0;
    std::mutex mu;
    std::condition_variable cv_work;  // workers wait for admissions
    std::condition_variable cv_done;  // clients wait for completions
    // submitted, not admitted: by (cells, id) for shortest-first admission and
    // by id (= arrival order) for the age limit
    std::set<std::pair<double, int64_t>> waiting;
    std::set<int64_t> waiting_by_age;
    std::deque<int64_t> admitted;     // admitted, not started
    std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
    size_t in_use = 0;  // bytes of admitted + resident requests
    int free_slots = 0;
    int64_t next_id = 1;
    bool stop = false;
    std::vector<std::thread> workers;
    // epoch mode (FP32 re-anchored form)
    bool epochs = false;
    int slots = 0;
    std::thread engine;
    cudaMemPool_t pool = nullptr;
    int64_t epochs_launched = 0;
    // statistics
    int64_t completed = 0, rejected = 0;
    double cells_done = 0.0;
};

namespace {

size_t result_bytes(int64_t PL) { return 16 * (size_t)PL + 512; }

double cells_of(int64_t n, int64_t m) {
    const double L = (double)std::max<int64_t>(n - m + 1 - m / 4 - 1, 0);
    return L * (L + 1) / 2;
}

// A waiting request that has waited this long is admitted before any other.
constexpr double kAgeLimitS = 2.0;

// Moves waiting requests to `admitted` while slots and memory allow.  The
// oldest request goes first once it has waited kAgeLimitS (and while it does
// not fit the memory left, nothing else is admitted); otherwise the one with
// the fewest cells among those that fit (ties: arrival order).
void admit_locked(mp_server* s) {
    const Clock::time_point now = Clock::now();
    while (!s->waiting.empty() && s->free_slots > 0) {
        auto fits = [&](const Request* q) { return s->in_use + q->need <= s->budget || s->in_use == 0; };
        Request* r = s->reqs[*s->waiting_by_age.begin()].get();  // the oldest
        if (std::chrono::duration<double>(now - r->submitted).count() >= kAgeLimitS) {
            if (!fits(r)) break;
        } else {
            // the fewest cells among those that fit; the first one nearly always
            // does (a request's memory grows with its length, as its cells do)
            r = nullptr;
            for (const auto& e : s->waiting) {
                Request* q = s->reqs[e.second].get();
                if (fits(q)) {
                    r = q;
                    break;
                }
            }
            if (!r) break;
        }
        s->waiting.erase({r->cells, r->id});
        s->waiting_by_age.erase(r->id);
        s->in_use += r->need;
        r->accounted = r->need;
        --s->free_slots;
        s->admitted.push_back(r->id);
        s->cv_work.notify_one();
    }
}

void worker_main(mp_server* s) {
    cudaSetDevice(s->device);
    cudaStream_t st;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    mp_context* ctx = nullptr;
    mp_context_create(s->device, 0, &ctx);
    for (;;) {
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || !s->admitted.empty(); });
            if (s->stop && s->admitted.empty()) break;
            r = s->reqs[s->admitted.front()].get();
            s->admitted.pop_front();
            r->started = Clock::now();
        }
        const int64_t n = (int64_t)r->series.size(), PL = r->PL;
        int rc = ctx ? MP_OK : MP_ERR_NO_DEVICE;
        // scratch and result from the server's pool (the request's `need`)
        const size_t scr = mp_selfjoin_scratch_bytes(n, r->m, s->precision);
        void* scratch = nullptr;
        if (rc == MP_OK &&
            (cudaMallocFromPoolAsync((void**)&r->d_d2, 8 * PL, s->pool, st) != cudaSuccess ||
             cudaMallocFromPoolAsync((void**)&r->d_idx, 8 * PL, s->pool, st) != cudaSuccess ||
             cudaMallocFromPoolAsync(&scratch, scr, s->pool, st) != cudaSuccess)) {
            cudaGetLastError();
            rc = MP_ERR_OUT_OF_MEMORY;
        }
        if (rc == MP_OK) {
            mpgpu::ctx_lend_scratch(ctx, scratch, scr);
            rc = mp_selfjoin(ctx, r->series.data(), n, r->m, -1, s->precision, s->reanchor_k, 0, 0,
                             0, r->d_d2, r->d_idx, st);
            mpgpu::ctx_lend_scratch(ctx, nullptr, 0);
        }
        if (scratch) cudaFreeAsync(scratch, st);
        if (rc != MP_OK) {
            if (r->d_d2) cudaFreeAsync(r->d_d2, st);
            if (r->d_idx) cudaFreeAsync(r->d_idx, st);
            r->d_d2 = nullptr;
            r->d_idx = nullptr;
            cudaStreamSynchronize(st);
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r->finished = Clock::now();
            r->status = rc;
            r->series.clear();
            r->series.shrink_to_fit();
            // scratch is released; a resident result keeps its share
            const size_t keep = (rc == MP_OK) ? result_bytes(PL) : 0;
            s->in_use -= r->accounted - keep;
            r->accounted = keep;
            ++s->free_slots;
            if (rc == MP_OK) {
                ++s->completed;
                s->cells_done += cells_of(n, r->m);
            }
            admit_locked(s);
        }
        s->cv_done.notify_all();
    }
    if (ctx) mp_context_destroy(ctx);
    cudaStreamDestroy(st);
}

// ---- epoch mode -------------------------------------------------------------

// Cells per epoch: about 4 ms of the FP32 tile kernel on a B200 -- short enough
// that a new request waits little, long enough that the launch tail (warps
// running out of tiles) stays a few percent.
constexpr double kEpochCells = 1.2e10;
constexpr int kEpochsInFlight = 2;

// Picks the epoch's slices: every request with tiles left first gets a
// minimum share (a quarter of the epoch split evenly), then the remaining
// budget goes to the requests with the fewest cells left.
std::vector<mpgpu::ServeSlice> choose_slices(std::vector<Request*>& act) {
    std::vector<mpgpu::ServeSlice> out;
    std::vector<Request*> open;
    for (Request* r : act)
        if (r->job.next_tile < r->job.ntiles) open.push_back(r);
    if (open.empty()) return out;
    auto tile_cells = [](const mpgpu::ServeJob& j) { return 256.0 * (double)j.K; };
    auto left_cells = [&](const Request* r) {
        return (double)(r->job.ntiles - r->job.next_tile) * tile_cells(r->job);
    };
    std::stable_sort(open.begin(), open.end(),
                     [&](const Request* a, const Request* b) { return left_cells(a) < left_cells(b); });
    std::vector<int64_t> give(open.size(), 0);
    double budget = kEpochCells;
    const double share = kEpochCells / (4.0 * (double)open.size());
    for (size_t i = 0; i < open.size(); ++i) {
        const mpgpu::ServeJob& j = open[i]->job;
        const int64_t left = j.ntiles - j.next_tile;
        const int64_t t = std::min<int64_t>(left, std::max<int64_t>(1, (int64_t)(share / tile_cells(j))));
        give[i] = t;
        budget -= (double)t * tile_cells(j);
    }
    for (size_t i = 0; i < open.size() && budget > 0; ++i) {
        const mpgpu::ServeJob& j = open[i]->job;
        const int64_t left = j.ntiles - j.next_tile - give[i];
        const int64_t t = std::min<int64_t>(left, (int64_t)(budget / tile_cells(j)));
        if (t <= 0) continue;
        give[i] += t;
        budget -= (double)t * tile_cells(j);
    }
    for (size_t i = 0; i < open.size(); ++i)
        if (give[i] > 0) out.push_back({&open[i]->job, open[i]->job.next_tile, give[i]});
    return out;
}

// Marks requests finished (their last epoch and finalisation are done).
void complete_locked(mp_server* s, const std::vector<Request*>& done, int status) {
    const Clock::time_point now = Clock::now();
    for (Request* r : done) {
        r->finished = now;
        r->status = status;
        const size_t keep = (status == MP_OK) ? mpgpu::serve_result_bytes(r->job.n, r->m) : 0;
        s->in_use -= r->accounted - keep;
        r->accounted = keep;
        ++s->free_slots;
        if (status == MP_OK) {
            ++s->completed;
            s->cells_done += r->job.cells;
        }
    }
    admit_locked(s);
}

void engine_main(mp_server* s) {
    cudaSetDevice(s->device);
    cudaStream_t st;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    mpgpu::ServeEpochBuffers eb;
    const cudaError_t be = mpgpu::serve_epoch_buffers_create(eb, s->slots);
    struct InFlight {
        cudaEvent_t ev;
        std::vector<Request*> finishing;
    };
    std::deque<InFlight> inflight;
    std::vector<Request*> active;  // prepared, tiles left to launch
    std::vector<cudaEvent_t> spare;
    auto retire_front = [&]() {
        InFlight f = std::move(inflight.front());
        inflight.pop_front();
        const int status = cudaEventSynchronize(f.ev) == cudaSuccess ? MP_OK : MP_ERR_CUDA;
        spare.push_back(f.ev);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            for (Request* r : f.finishing) {
                r->series.clear();
                r->series.shrink_to_fit();
            }
            complete_locked(s, f.finishing, status);
        }
        s->cv_done.notify_all();
    };
    for (;;) {
        std::vector<Request*> fresh;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            const bool busy = !inflight.empty() ||
                              std::any_of(active.begin(), active.end(), [](const Request* r) {
                                  return r->job.next_tile < r->job.ntiles;
                              });
            if (!busy)
                s->cv_work.wait(lk, [&] { return s->stop || !s->admitted.empty(); });
            if (s->stop && s->admitted.empty() && !busy) break;
            while (!s->admitted.empty()) {
                Request* r = s->reqs[s->admitted.front()].get();
                s->admitted.pop_front();
                r->started = Clock::now();
                fresh.push_back(r);
            }
        }
        // new requests: device buffers from the pool, series in, preparation
        std::vector<Request*> failed, finishing;
        for (Request* r : fresh) {
            cudaError_t e = be;
            if (e == cudaSuccess)
                e = mpgpu::serve_prepare(r->job, r->series.data(), (int64_t)r->series.size(), r->m,
                                         s->reanchor_k, s->pool, st);
            if (e != cudaSuccess) {
                cudaGetLastError();
                mpgpu::serve_release_result(r->job, st);
                failed.push_back(r);
                continue;
            }
            r->d_d2 = r->job.d2;
            r->d_idx = r->job.idx;
            if (r->job.ntiles == 0) {  // no diagonal outside the exclusion zone
                if (mpgpu::serve_finalize(r->job, st) != cudaSuccess) {
                    cudaGetLastError();
                    mpgpu::serve_release_result(r->job, st);
                    r->d_d2 = nullptr;
                    r->d_idx = nullptr;
                    failed.push_back(r);
                } else {
                    finishing.push_back(r);
                }
                continue;
            }
            active.push_back(r);
        }
        if (!failed.empty()) {
            cudaStreamSynchronize(st);
            {
                std::lock_guard<std::mutex> lk(s->mu);
                for (Request* r : failed) {
                    r->d_d2 = nullptr;
                    r->d_idx = nullptr;
                }
                complete_locked(s, failed, MP_ERR_OUT_OF_MEMORY);
            }
            s->cv_done.notify_all();
        }
        // one epoch over slices of every active request
        std::vector<mpgpu::ServeSlice> slices = choose_slices(active);
        if (!slices.empty()) {
            mpgpu::serve_launch_epoch(eb, (int)(s->epochs_launched % mpgpu::ServeEpochBuffers::kRing),
                                      slices, st);
            ++s->epochs_launched;
            for (const mpgpu::ServeSlice& sl : slices) sl.job->next_tile += sl.count;
            for (auto it = active.begin(); it != active.end();) {
                Request* r = *it;
                if (r->job.next_tile >= r->job.ntiles) {
                    mpgpu::serve_finalize(r->job, st);
                    finishing.push_back(r);
                    it = active.erase(it);
                } else {
                    ++it;
                }
            }
        }
        if (!finishing.empty() || !slices.empty()) {
            cudaEvent_t ev;
            if (!spare.empty()) {
                ev = spare.back();
                spare.pop_back();
            } else {
                cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            }
            cudaEventRecord(ev, st);
            inflight.push_back({ev, std::move(finishing)});
        }
        // keep kEpochsInFlight epochs queued; drain when there is nothing to add
        while ((int)inflight.size() > kEpochsInFlight || (slices.empty() && !inflight.empty()))
            retire_front();
    }
    while (!inflight.empty()) retire_front();
    cudaStreamSynchronize(st);
    for (cudaEvent_t e : spare) cudaEventDestroy(e);
    mpgpu::serve_epoch_buffers_destroy(eb);
    cudaStreamDestroy(st);
}

}  // namespace

extern "C" {

int mp_server_create(int device, size_t mem_budget_bytes, int slots, int precision,
                     int64_t reanchor_k, mp_server** out) {
    if (!out || slots < 1 || mem_budget_bytes == 0) return MP_ERR_INVALID_ARG;
    if (precision != MP_PREC_FP64 && precision != MP_PREC_FP32_REANCHOR &&
        precision != MP_PREC_FP32_GUARDED)
        return MP_ERR_INVALID_ARG;
    mp_context* probe = nullptr;
    const int rc = mp_context_create(device, 0, &probe);
    if (rc != MP_OK) return rc;
    mp_context_destroy(probe);
    mp_server* s = new mp_server();
    s->device = device;
    s->budget = mem_budget_bytes;
    s->precision = precision;
    s->reanchor_k = reanchor_k;
    s->free_slots = slots;
    s->slots = slots;
    s->epochs = precision == MP_PREC_FP32_REANCHOR;
    // a pool of the server's own that keeps what it has been given (no release
    // to the driver between requests); the budget bounds it.  Every device
    // buffer of a request (scratch and result) comes from it.
    cudaSetDevice(device);
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&s->pool, &props) != cudaSuccess) {
        cudaGetLastError();
        delete s;
        return MP_ERR_CUDA;
    }
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (s->epochs) {
        s->engine = std::thread(engine_main, s);
    } else {
        for (int i = 0; i < slots; ++i) s->workers.emplace_back(worker_main, s);
    }
    *out = s;
    return MP_OK;
}

int mp_server_submit(mp_server* s, const double* A, int64_t n, int64_t m, int64_t* ticket) {
    if (!s || !A || !ticket || m < 2 || n < m) return MP_ERR_INVALID_ARG;
    auto r = std::make_unique<Request>();
    r->series.assign(A, A + n);
    r->m = m;
    r->PL = n - m + 1;
    r->cells = cells_of(n, m);
    r->need = s->epochs ? mpgpu::serve_scratch_bytes(n, m) + mpgpu::serve_result_bytes(n, m)
                        : mp_selfjoin_scratch_bytes(n, m, s->precision) + result_bytes(n - m + 1);
    r->submitted = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    *ticket = r->id;
    if (r->need > s->budget) {
        r->status = MP_ERR_BUDGET;
        r->finished = r->submitted;
        ++s->rejected;
        s->reqs[r->id] = std::move(r);
        return MP_ERR_BUDGET;
    }
    const int64_t id = r->id;
    s->reqs[id] = std::move(r);
    s->waiting.insert({s->reqs[id]->cells, id});
    s->waiting_by_age.insert(id);
    admit_locked(s);
    return MP_OK;
}

// 0 = pending, 1 = finished (status then holds the result's status).
int mp_server_poll(mp_server* s, int64_t ticket, int* status) {
    if (!s) return MP_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return MP_ERR_INVALID_ARG;
    if (status) *status = it->second->status;
    return it->second->status >= 0 ? 1 : 0;
}

int mp_server_collect(mp_server* s, int64_t ticket, double* dist2_out, int64_t* idx_out,
                      double* latency_s, double* queue_s) {
    if (!s) return MP_ERR_INVALID_ARG;
    Request* r = nullptr;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return MP_ERR_INVALID_ARG;
        r = it->second.get();
        s->cv_done.wait(lk, [&] { return r->status >= 0; });
        if (r->collected) return MP_ERR_INVALID_ARG;
        r->collected = true;
    }
    int rc = r->status;
    if (latency_s)
        *latency_s = std::chrono::duration<double>(r->finished - r->submitted).count();
    if (queue_s)
        *queue_s = rc == MP_ERR_BUDGET
                       ? 0.0
                       : std::chrono::duration<double>(r->started - r->submitted).count();
    if (r->d_d2) {
        // a private stream: no device-wide synchronisation while others run
        cudaSetDevice(s->device);
        cudaStream_t st;
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (rc == MP_OK) {
            if ((dist2_out &&
                 cudaMemcpyAsync(dist2_out, r->d_d2, 8 * r->PL, cudaMemcpyDeviceToHost, st) != cudaSuccess) ||
                (idx_out &&
                 cudaMemcpyAsync(idx_out, r->d_idx, 8 * r->PL, cudaMemcpyDeviceToHost, st) != cudaSuccess)) {
                cudaGetLastError();
                rc = MP_ERR_CUDA;
            }
        }
        cudaFreeAsync(r->d_d2, st);
        cudaFreeAsync(r->d_idx, st);
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->in_use -= r->accounted;
        s->reqs.erase(ticket);
        admit_locked(s);
    }
    return rc;
}

int mp_server_stats(mp_server* s, int64_t* completed, int64_t* rejected, int64_t* waiting,
                    int64_t* running, double* cells, size_t* bytes_in_use) {
    if (!s) return MP_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (completed) *completed = s->completed;
    if (rejected) *rejected = s->rejected;
    if (waiting) *waiting = (int64_t)s->waiting.size();
    if (running) *running = (int64_t)s->slots - s->free_slots;
    if (cells) *cells = s->cells_done;
    if (bytes_in_use) *bytes_in_use = s->in_use;
    return MP_OK;
}

int mp_server_destroy(mp_server* s) {
    if (!s) return MP_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->waiting.clear();
        s->waiting_by_age.clear();
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    if (s->engine.joinable()) s->engine.join();
    cudaSetDevice(s->device);
    cudaStream_t st;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    for (auto& kv : s->reqs) {
        if (kv.second->d_d2) cudaFreeAsync(kv.second->d_d2, st);
        if (kv.second->d_idx) cudaFreeAsync(kv.second->d_idx, st);
    }
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return MP_OK;
}

}  // extern "C"
