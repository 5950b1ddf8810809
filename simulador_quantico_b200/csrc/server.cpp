// Serving mode: continuous batching of circuits on one GPU.
//
// Clients submit circuits at any time.  hgm_server_submit copies the circuit
// and returns; a few planner threads plan and upload submitted circuits while
// earlier requests run (hgm_server_submit_plan takes a plan built
// beforehand).  One worker thread
//   * admits planned requests in the order their plans are ready, while a
//     slot is free and the request's state bytes (16*2^n FP64, 8*2^n FP32)
//     fit the HBM budget (a request larger than the whole budget is refused);
//   * gives each admitted request a slot -- a CUDA stream with its own
//     reduction scratch -- and a state buffer from the server's cache of
//     device buffers, initialises it, queues the plan's passes, an FP64 norm
//     and (if asked) the marginal argmax, copies those few numbers to pinned
//     host memory and records an event;
//   * feeds each slot's passes in chunks (at most two chunks ahead of the
//     GPU) and polls the slots' events; a finished request records its
//     completion time, returns (or keeps) its state buffer, hands its plan
//     to a planner thread for release and frees the slot for the next one.
// State sizes are powers of two, so finished states are kept by size and
// handed to the next request of that size: after warm-up the worker makes
// no allocation calls.  (Allocating from the stream-ordered pool per request
// blocked the worker, and with it every slot, for up to half a second when
// the pool had to map memory for a 1-2 GiB state.)  New buffers are
// cudaMalloc'ed while admitted plus cached bytes stay within the budget;
// cached buffers of other sizes are freed first when they would not.  Plans
// the planner threads build take their device memory from a cache of
// power-of-two blocks (PlanMemory), so serving from host circuits makes no
// allocation calls once warm either.
// Requests on different slots run concurrently on the device; new requests
// are admitted while earlier ones are still executing.  A request's result
// does not depend on what else runs: it uses its own plan, state and scratch
// and fixed-order reductions.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "hgm_internal.h"

namespace hgm {

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
    int64_t id = 0;
    int n = 0;
    int64_t init_index = 0;
    uint64_t result_mask = 0;
    std::vector<Op> ops;          // hgm_server_submit: the circuit, until a planner thread plans it
    hgm_plan_opts popts{};
    std::unique_ptr<Plan> owned;  // planned by a planner thread
    const Plan *plan = nullptr;   // owned, or borrowed (hgm_server_submit_plan)
    int64_t bytes = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
    State state;  // device state (pool memory)
    int status = HGM_OK;
    double norm = 0, pmax = 0;
    int64_t argmax = -1;
    bool leased = false;  // `plan` is borrowed and leased (hgm_server_submit_plan)
    ~Request() {
        if (leased) plan_unlease(plan);
    }
};

// Passes are queued on a slot's stream in chunks, at most two chunks ahead
// of the GPU: a long plan (a Grover circuit is thousands of passes) then
// neither fills the launch queue -- where the worker would block, and every
// other slot with it -- nor starves the slots admitted after it.
constexpr int64_t kChunkLaunches = 16;

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    cudaEvent_t chunk[2] = {nullptr, nullptr};
    int chunks_in_flight = 0, chunk_next = 0;
    PlanCursor cursor;
    int64_t total = 0;   // launches of the request's plan
    bool tail = false;   // reductions and result copy queued (s.done recorded)
    double *partials = nullptr;
    long long *ibest = nullptr;
    double *dres = nullptr;   // 4 doubles: norm (2 slots), argmax probability and index
    double *hres = nullptr;   // pinned, 6 doubles: dres, then a chained run's error word
    Request *req = nullptr;
};

}  // namespace

// Device buffers for request states, cached by size.  Worker and client
// threads both return buffers, so it has its own lock.
struct StateCache {
    std::mutex mu;
    std::map<int64_t, std::vector<void *>> free_by_size;
    int64_t cached = 0;  // bytes held in free_by_size

    // A buffer of `bytes`; `others` = bytes the server holds outside the
    // cache (admitted states, this one included), `budget` their limit.
    int acquire(int64_t bytes, int64_t others, int64_t budget, void **out) {
        std::lock_guard<std::mutex> lk(mu);
        auto &v = free_by_size[bytes];
        if (!v.empty()) {
            *out = v.back();
            v.pop_back();
            cached -= bytes;
            return HGM_OK;
        }
        // make room: free cached buffers, largest first, while over budget
        while (others + cached > budget && cached > 0) evict_largest();
        cudaError_t e = cudaMalloc(out, (size_t)bytes);
        if (e != cudaSuccess && cached > 0) {
            cudaGetLastError();
            while (cached > 0) evict_largest();
            e = cudaMalloc(out, (size_t)bytes);
        }
        return e == cudaSuccess ? HGM_OK : fail(HGM_ERR_NOMEM, "request state: %s", cudaGetErrorString(e));
    }
    // The GPU must be done with the buffer.
    void release(void *p, int64_t bytes) {
        std::lock_guard<std::mutex> lk(mu);
        free_by_size[bytes].push_back(p);
        cached += bytes;
    }
    void evict_largest() {
        for (auto it = free_by_size.rbegin(); it != free_by_size.rend(); ++it)
            if (!it->second.empty()) {
                cudaFree(it->second.back());
                it->second.pop_back();
                cached -= it->first;
                return;
            }
        cached = 0;
    }
    ~StateCache() {
        for (auto &kv : free_by_size)
            for (void *p : kv.second) cudaFree(p);
    }
};

// Device memory for the plans the planner threads upload, recycled by
// power-of-two size class (a plan's records are a few tens of KB).
// cudaMalloc and cudaFree take the device's allocation lock and cudaFree
// can wait on running work, so freeing a finished request's plan while
// other slots run stalled them all; recycled blocks avoid both calls.
// Every block it hands out is its own cudaMalloc of the class size, and a
// block comes back only as the pointer and class it went out with (`live`
// holds the blocks out): a pointer into the middle of a block, or one freed
// twice, is refused rather than entered in a free list, where it would later
// be handed out as a block overlapping a live one.
struct PlanMemory : DevAllocator {
    std::mutex mu;
    std::map<size_t, std::vector<void *>> free_by_class;
    std::map<void *, size_t> live;
    static size_t size_class(size_t b) {
        size_t c = 256;
        while (c < b) c <<= 1;
        return c;
    }
    cudaError_t alloc(void **p, size_t bytes) override {
        const size_t c = size_class(bytes);
        std::lock_guard<std::mutex> lk(mu);
        auto &v = free_by_class[c];
        if (!v.empty()) {
            *p = v.back();
            v.pop_back();
        } else {
            cudaError_t e = cudaMalloc(p, c);
            if (e != cudaSuccess) return e;
        }
        live[*p] = c;
        return cudaSuccess;
    }
    // The GPU must be done with the block.
    void free(void *p, size_t bytes) override {
        std::lock_guard<std::mutex> lk(mu);
        auto it = live.find(p);
        if (it == live.end() || it->second != size_class(bytes)) {
            set_error("plan memory: a block was returned that this cache did not hand out");
            return;
        }
        live.erase(it);
        free_by_class[size_class(bytes)].push_back(p);
    }
    ~PlanMemory() {
        for (auto &kv : free_by_class)
            for (void *p : kv.second) cudaFree(p);
        for (auto &kv : live) cudaFree(kv.first);
    }
};

struct Server {
    // declared first, destroyed last: every plan below returns its blocks here
    PlanMemory plan_mem;
    hgm_server_opts opts;
    StateCache cache;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request *> queue;
    std::vector<Slot> slots;
    std::map<int64_t, Request *> kept;      // finished requests whose states are kept
    std::deque<hgm_result> results;
    std::condition_variable results_cv;
    int64_t bytes_in_use = 0;
    int64_t next_id = 1;
    std::atomic<bool> stop{false};
    std::thread worker;
    std::deque<Request *> to_plan;   // submitted circuits waiting for a planner thread
    // plans of finished requests, released by a planner thread
    std::vector<std::unique_ptr<Plan>> to_reap;
    std::condition_variable plan_cv;
    std::vector<std::thread> planners;
    int planning = 0;                // circuits being planned
    int inflight = 0;
    int error = HGM_OK;
    std::string error_msg;  // the worker's message for `error`, reported by hgm_server_poll

    ~Server() {
        {
            // under the mutex: a thread between its predicate check and its
            // wait would otherwise miss the wake-up and never return
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        plan_cv.notify_all();
        cv.notify_all();
        for (std::thread &t : planners)
            if (t.joinable()) t.join();
        if (worker.joinable()) worker.join();
        for (Request *r : to_plan) delete r;
        for (Slot &s : slots) {
            if (s.stream) cudaStreamSynchronize(s.stream);
            if (s.req) {
                if (s.req->state.d) cudaFree(s.req->state.d);
                delete s.req;
            }
            if (s.partials) cudaFree(s.partials);
            if (s.ibest) cudaFree(s.ibest);
            if (s.dres) cudaFree(s.dres);
            if (s.hres) cudaFreeHost(s.hres);
            if (s.done) cudaEventDestroy(s.done);
            for (cudaEvent_t ev : s.chunk)
                if (ev) cudaEventDestroy(ev);
            if (s.stream) cudaStreamDestroy(s.stream);
        }
        for (Request *r : queue) delete r;
        for (auto &kv : kept) {
            if (kv.second->state.d) cudaFree(kv.second->state.d);
            delete kv.second;
        }
    }

    void finish(Slot &s) {
        Request *r = s.req;
        r->t_done = now_s();
        r->norm = s.hres[0];
        uint64_t chain_err = 0;
        memcpy(&chain_err, s.hres + 4, sizeof chain_err);
        if (chain_err && r->status == HGM_OK)
            r->status = fail(HGM_ERR_TIMEOUT, "request %lld: a chained pass gave up waiting", (long long)r->id);
        if (r->result_mask) {
            r->pmax = s.hres[2];
            r->argmax = (int64_t)s.hres[3];
        }
        hgm_result res;
        res.id = r->id;
        res.status = r->status;
        res.qubits = r->n;
        res.latency_s = r->t_done - r->t_submit;
        res.queue_s = r->t_admit - r->t_submit;
        res.exec_s = r->t_done - r->t_admit;
        res.norm = r->norm;
        res.argmax = r->argmax;
        res.pmax = r->pmax;
        if (opts.keep_states) {
            std::lock_guard<std::mutex> lk(mu);
            kept[r->id] = r;
        } else {
            if (r->state.d) cache.release(r->state.d, r->bytes);  // s.done has completed: the GPU is done with it
            r->state.d = nullptr;
            std::lock_guard<std::mutex> lk(mu);
            bytes_in_use -= r->bytes;
            if (r->owned) {
                to_reap.push_back(std::move(r->owned));
                plan_cv.notify_one();
            }
            delete r;
        }
        s.req = nullptr;
        {
            std::lock_guard<std::mutex> lk(mu);
            results.push_back(res);
            inflight--;
        }
        results_cv.notify_all();
    }

    int start(Slot &s, Request *r) {
        r->t_admit = now_s();
        s.req = r;
        int64_t held;
        {
            std::lock_guard<std::mutex> lk(mu);
            held = bytes_in_use;
        }
        int arc = cache.acquire(r->bytes, held, opts.budget_bytes, &r->state.d);
        if (arc) return arc;
        r->state.qubits = r->n;
        r->state.precision = opts.precision;
        s.cursor = PlanCursor();
        s.total = plan_launches(r->plan, 1);
        s.chunks_in_flight = 0;
        s.tail = false;
        s.hres[4] = 0.0;  // the error word of a chained run is copied here behind it
        int rc = launch_set_basis(&r->state, r->init_index, s.stream);
        return rc ? rc : feed(s);
    }

    // Queues the slot's next chunks (while fewer than two are in flight) and,
    // after the last pass, the reductions, the result copy and s.done.
    int feed(Slot &s) {
        Request *r = s.req;
        while (!s.tail && s.chunks_in_flight < 2) {
            if (s.cursor.next == 0 && s.total > 1 && chain_eligible(r->plan, 1)) {
                // a small state: every pass in one persistent launch
                int rc = launch_plan_chain(&r->state, r->plan, 1, s.stream);
                if (rc) return rc;
                cudaMemcpyAsync(s.hres + 4, chain_error_word(r->plan), sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                s.stream);
                s.cursor.next = s.total;
            }
            if (s.cursor.next < s.total) {
                int rc = launch_plan_steps(&r->state, r->plan, 1, &s.cursor, kChunkLaunches, s.stream);
                if (rc) return rc;
                cudaError_t e = cudaEventRecord(s.chunk[s.chunk_next], s.stream);
                if (e != cudaSuccess) return fail(HGM_ERR_CUDA, "event record: %s", cudaGetErrorString(e));
                s.chunk_next ^= 1;
                s.chunks_in_flight++;
            }
            if (s.cursor.next >= s.total) {
                int rc = launch_norm_async(&r->state, s.partials, s.dres, s.stream);
                if (!rc && r->result_mask)
                    rc = launch_argmax_async(&r->state, r->result_mask, s.partials, s.ibest, s.dres + 2, s.stream);
                if (rc) return rc;
                cudaMemcpyAsync(s.hres, s.dres, 4 * sizeof(double), cudaMemcpyDeviceToHost, s.stream);
                cudaError_t e = cudaEventRecord(s.done, s.stream);
                if (e != cudaSuccess) return fail(HGM_ERR_CUDA, "event record: %s", cudaGetErrorString(e));
                s.tail = true;
            }
        }
        return HGM_OK;
    }

    int device = 0;

    // Planner thread: plans and uploads submitted circuits, then hands them to
    // the worker.  A request is admitted once its plan is ready, so a quick
    // circuit is not held behind a slow one.
    void plan_loop() {
        cudaSetDevice(device);
        for (;;) {
            Request *r = nullptr;
            std::vector<std::unique_ptr<Plan>> reap;
            {
                std::unique_lock<std::mutex> lk(mu);
                while (!stop && to_plan.empty() && to_reap.empty())
                    plan_cv.wait_for(lk, std::chrono::milliseconds(100));
                if (stop) return;
                reap.swap(to_reap);
                if (!to_plan.empty()) {
                    r = to_plan.front();
                    to_plan.pop_front();
                    planning++;
                }
            }
            reap.clear();  // returns the finished requests' plan memory
            if (!r) continue;
            r->owned.reset(new Plan());
            r->owned->allocator = &plan_mem;
            int rc = build_plan(r->ops, r->n, r->popts, r->owned.get());
            if (!rc) rc = upload_plan(r->owned.get());
            std::vector<Op>().swap(r->ops);
            r->plan = r->owned.get();
            std::lock_guard<std::mutex> lk(mu);
            planning--;
            if (rc) {  // never runs: its result carries the planning status
                hgm_result res{};
                res.id = r->id;
                res.status = rc;
                res.qubits = r->n;
                res.latency_s = now_s() - r->t_submit;
                res.argmax = -1;
                results.push_back(res);
                delete r;
                results_cv.notify_all();
            } else {
                queue.push_back(r);
                cv.notify_all();
            }
        }
    }

    void enqueue(Request *r, int64_t *id) {
        {
            std::lock_guard<std::mutex> lk(mu);
            r->id = next_id++;
            if (id) *id = r->id;
            queue.push_back(r);
        }
        cv.notify_all();
    }

    void loop() {
        cudaSetDevice(device);
        while (!stop) {
            bool progress = false;
            // completions
            for (Slot &s : slots) {
                if (!s.req) continue;
                cudaError_t q;
                if (!s.tail) {
                    // retire the oldest chunk if it has run, then queue more
                    const int oldest = (s.chunk_next + 2 - s.chunks_in_flight) & 1;
                    q = s.chunks_in_flight ? cudaEventQuery(s.chunk[oldest]) : cudaSuccess;
                    if (q == cudaSuccess) {
                        if (s.chunks_in_flight) s.chunks_in_flight--;
                        int rc = feed(s);
                        if (rc) {
                            s.req->status = rc;
                            cudaStreamSynchronize(s.stream);
                            finish(s);
                        }
                        progress = true;
                        continue;
                    }
                    if (q == cudaErrorNotReady) continue;
                    // a chunk failed: reported below like a failed request
                } else {
                    q = cudaEventQuery(s.done);  // s.done belongs to this request once the tail is queued
                }
                if (q == cudaSuccess) {
                    finish(s);
                    progress = true;
                } else if (q != cudaErrorNotReady) {
                    s.req->status = HGM_ERR_CUDA;
                    {
                        std::lock_guard<std::mutex> lk(mu);
                        error_msg = "request " + std::to_string(s.req->id) + " (" + std::to_string(s.req->n) +
                                    " qubits) execution: " + cudaGetErrorString(q);
                        error = HGM_ERR_CUDA;
                    }
                    finish(s);
                    progress = true;
                }
            }
            // admissions: in arrival order (the head waits for budget), or the
            // queued request with the most work that fits
            for (Slot &s : slots) {
                if (s.req) continue;
                Request *r = nullptr;
                {
                    std::lock_guard<std::mutex> lk(mu);
                    if (queue.empty()) break;
                    auto pick = queue.begin();
                    if (opts.order == HGM_ORDER_WORK_FIRST) {
                        pick = queue.end();
                        double best = -1.0;
                        for (auto it = queue.begin(); it != queue.end(); ++it) {
                            if (bytes_in_use + (*it)->bytes > opts.budget_bytes) continue;
                            const Plan *pl = (*it)->plan;
                            const double w = (double)(*it)->bytes * (pl->small ? 1.0 : (double)pl->passes.size());
                            if (w > best) {
                                best = w;
                                pick = it;
                            }
                        }
                        if (pick == queue.end()) break;
                    } else if (bytes_in_use + queue.front()->bytes > opts.budget_bytes) {
                        break;
                    }
                    r = *pick;
                    queue.erase(pick);
                    bytes_in_use += r->bytes;
                    inflight++;
                }
                int rc = start(s, r);
                if (rc) {
                    r->status = rc;
                    cudaStreamSynchronize(s.stream);
                    finish(s);
                }
                progress = true;
            }
            if (!progress) {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait_for(lk, std::chrono::microseconds(inflight ? 20 : 500));
            }
        }
    }
};

}  // namespace hgm

using namespace hgm;

extern "C" {

void hgm_server_default_opts(hgm_server_opts *o, int precision) {
    o->precision = precision;
    o->budget_bytes = (int64_t)150 << 30;
    o->max_inflight = 32;  // one per hardware queue (hgm_init asks for 32)
    o->keep_states = 0;
    o->warp_bits = -1;
    o->order = HGM_ORDER_ARRIVAL;
}

int hgm_server_create(const hgm_server_opts *opts, hgm_server **out) {
    if (!opts || !out) return fail(HGM_ERR_INVALID, "null argument");
    if (opts->max_inflight < 1 || opts->max_inflight > 256) return fail(HGM_ERR_INVALID, "max_inflight outside 1..256");
    if (opts->order != HGM_ORDER_ARRIVAL && opts->order != HGM_ORDER_WORK_FIRST)
        return fail(HGM_ERR_INVALID, "unknown admission order %d", opts->order);
    if (!default_stream()) return HGM_ERR_CUDA;
    std::unique_ptr<Server> s(new Server());
    s->opts = *opts;
    s->slots.resize(opts->max_inflight);
    for (Slot &sl : s->slots) {
        cudaError_t e;
        if ((e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&sl.chunk[0], cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&sl.chunk[1], cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaMalloc(&sl.partials, 2 * REDUCE_SCRATCH_BLOCKS * sizeof(double))) != cudaSuccess ||
            (e = cudaMalloc(&sl.ibest, REDUCE_SCRATCH_BLOCKS * sizeof(long long))) != cudaSuccess ||
            (e = cudaMalloc(&sl.dres, 4 * sizeof(double))) != cudaSuccess ||
            (e = cudaMallocHost(&sl.hres, 6 * sizeof(double))) != cudaSuccess)
            return fail(HGM_ERR_CUDA, "server slot: %s", cudaGetErrorString(e));
    }
    cudaGetDevice(&s->device);
    Server *raw = s.get();
    s->worker = std::thread([raw] { raw->loop(); });
    const unsigned hw = std::thread::hardware_concurrency();
    const int np = (int)std::max(1u, std::min(8u, hw / 2));
    for (int i = 0; i < np; i++) s->planners.emplace_back([raw] { raw->plan_loop(); });
    *out = reinterpret_cast<hgm_server *>(s.release());
    return HGM_OK;
}

void hgm_server_free(hgm_server *s) { delete reinterpret_cast<Server *>(s); }

int hgm_server_submit(hgm_server *ss, const hgm_circuit *c, int qubits, int64_t init_index, uint64_t result_mask,
                      int64_t *id) {
    Server *s = reinterpret_cast<Server *>(ss);
    if (!s || !c) return fail(HGM_ERR_INVALID, "null argument");
    if (init_index < 0 || init_index >= (int64_t(1) << qubits)) return fail(HGM_ERR_INVALID, "initial index outside state");
    std::unique_ptr<Request> r(new Request());
    r->t_submit = now_s();
    r->n = qubits;
    r->init_index = init_index;
    r->result_mask = result_mask;
    r->bytes = (int64_t(1) << qubits) * (s->opts.precision == HGM_F64 ? 16 : 8);
    if (r->bytes > s->opts.budget_bytes)
        return fail(HGM_ERR_BUSY, "state of %lld bytes exceeds the %lld-byte budget", (long long)r->bytes,
                    (long long)s->opts.budget_bytes);
    hgm_plan_default_opts(&r->popts, s->opts.precision);
    r->popts.warp_bits = s->opts.warp_bits;
    r->ops = reinterpret_cast<const Circuit *>(c)->ops;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        if (id) *id = r->id;
        s->to_plan.push_back(r.release());
    }
    s->plan_cv.notify_one();
    return HGM_OK;
}

int hgm_server_submit_plan(hgm_server *ss, const hgm_plan *pp, int64_t init_index, uint64_t result_mask,
                           int64_t *id) {
    Server *s = reinterpret_cast<Server *>(ss);
    const Plan *p = reinterpret_cast<const Plan *>(pp);
    if (!s || !p) return fail(HGM_ERR_INVALID, "null argument");
    if (p->precision != s->opts.precision) return fail(HGM_ERR_INVALID, "plan precision differs from the server's");
    const int qubits = p->qubits;
    if (init_index < 0 || init_index >= (int64_t(1) << qubits)) return fail(HGM_ERR_INVALID, "initial index outside state");
    std::unique_ptr<Request> r(new Request());
    r->t_submit = now_s();
    r->n = qubits;
    r->init_index = init_index;
    r->result_mask = result_mask;
    r->bytes = (int64_t(1) << qubits) * (s->opts.precision == HGM_F64 ? 16 : 8);
    if (r->bytes > s->opts.budget_bytes)
        return fail(HGM_ERR_BUSY, "state of %lld bytes exceeds the %lld-byte budget", (long long)r->bytes,
                    (long long)s->opts.budget_bytes);
    // a plan is uploaded on first use; do it here, on the calling thread
    const int rc = upload_plan(const_cast<Plan *>(p));
    if (rc) return rc;
    r->plan = p;
    plan_lease(p);  // a plan freed while the request is queued or running waits for it
    r->leased = true;
    s->enqueue(r.release(), id);
    return HGM_OK;
}

int hgm_server_poll(hgm_server *ss, hgm_result *out, int max, int *n, int wait_ms) {
    Server *s = reinterpret_cast<Server *>(ss);
    if (!s || !out || !n) return fail(HGM_ERR_INVALID, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->results.empty() && wait_ms > 0)
        s->results_cv.wait_for(lk, std::chrono::milliseconds(wait_ms), [s] { return !s->results.empty(); });
    int k = 0;
    while (k < max && !s->results.empty()) {
        out[k++] = s->results.front();
        s->results.pop_front();
    }
    *n = k;
    if (s->error) return fail(s->error, "%s", s->error_msg.c_str());
    return HGM_OK;
}

int hgm_server_pending(hgm_server *ss, int *queued, int *inflight, int64_t *bytes_in_use) {
    Server *s = reinterpret_cast<Server *>(ss);
    if (!s) return fail(HGM_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (queued) *queued = (int)(s->to_plan.size() + s->planning + s->queue.size());
    if (inflight) *inflight = s->inflight;
    if (bytes_in_use) *bytes_in_use = s->bytes_in_use;
    return HGM_OK;
}

hgm_state *hgm_server_result_state(hgm_server *ss, int64_t id) {
    Server *s = reinterpret_cast<Server *>(ss);
    if (!s) return nullptr;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->kept.find(id);
    if (it == s->kept.end()) {
        fail(HGM_ERR_INVALID, "request %lld has no kept state", (long long)id);
        return nullptr;
    }
    it->second->state.owned = false;
    return reinterpret_cast<hgm_state *>(&it->second->state);
}

int hgm_server_release(hgm_server *ss, int64_t id) {
    Server *s = reinterpret_cast<Server *>(ss);
    if (!s) return fail(HGM_ERR_INVALID, "null server");
    Request *r = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->kept.find(id);
        if (it == s->kept.end()) return fail(HGM_ERR_INVALID, "request %lld has no kept state", (long long)id);
        r = it->second;
        s->kept.erase(it);
        s->bytes_in_use -= r->bytes;
    }
    // the caller may still have work on the library stream that reads it
    cudaStreamSynchronize((cudaStream_t)default_stream());
    if (r->state.d) s->cache.release(r->state.d, r->bytes);
    delete r;
    s->cv.notify_all();
    return HGM_OK;
}

}  // extern "C"
