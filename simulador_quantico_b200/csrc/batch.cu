// Batched mode: many independent circuits of uneven size in one persistent
// kernel, replayed from a CUDA graph.
//
// Every circuit is planned for the same register tile (R, W).  A circuit
// whose state is smaller than one tile (n < 5+R+W) becomes one "small" task:
// a CTA loads the whole state into shared memory and applies its gates one
// by one.  A larger circuit becomes one task per pass, each of 2^(n-K)
// tiles.  Tasks are laid out wave by wave (pass 0 of every circuit, then
// pass 1, ...), and the CTAs of one persistent grid claim tiles in that
// order from a global counter.  A tile of pass p may start only when every
// tile of pass p-1 of the same circuit is done: the claiming thread spins on
// that task's completion counter with a time limit (2 s of %globaltimer by
// default; the limit is a field of the task), after which it sets an error
// flag and the CTA skips the tile.  Because a
// tile only ever waits for tiles claimed before it, and a claimed tile is
// already held by a running CTA, the queue always makes progress, whether
// or not all CTAs are resident.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "kernels.cuh"

namespace hgm {

struct BatchTask {
    PassArgs pa;            // pass arguments (tiled tasks)
    void *state;            // the circuit's state in the batch arena
    long long tile_begin;   // first global item of this task
    int32_t ntiles;
    int32_t dep;            // task that must be complete first, -1 if none
    uint32_t dep_need;      // completions of `dep` to wait for (its tile count)
    unsigned long long wait_ns;  // limit of that wait
    int32_t small;          // 1: whole circuit in shared memory
    int32_t n;              // qubits
    const void *small_ops;  // SmallOp<Real>[] for small tasks
    long long n_small_ops;
};

constexpr unsigned long long BATCH_WAIT_LIMIT_NS = 2000000000ull;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <typename Real>
__device__ __forceinline__ void small_task(typename V2<Real>::T *__restrict__ state, int n,
                                           const SmallOp<Real> *__restrict__ ops, long long n_ops,
                                           typename V2<Real>::T *sm) {
    using A2 = typename V2<Real>::T;
    const int N = 1 << n, half = N >> 1;
    for (int i = threadIdx.x; i < N; i += blockDim.x) sm[i] = __ldcg(state + i);
    __syncthreads();
    for (long long k = 0; k < n_ops; k++) {
        const SmallOp<Real> &o = ops[k];
        const int t = o.target;
        const uint32_t cm = o.cmask, cv = o.cval;
        const Real m0r = o.m[0], m0i = o.m[1], m1r = o.m[2], m1i = o.m[3];
        const Real m2r = o.m[4], m2i = o.m[5], m3r = o.m[6], m3i = o.m[7];
        for (int p = threadIdx.x; p < half; p += blockDim.x) {
            const int i0 = ((p >> t) << (t + 1)) | (p & ((1 << t) - 1));
            const int i1 = i0 | (1 << t);
            if (((uint32_t)i0 & cm) != cv) continue;
            const A2 x = sm[i0], y = sm[i1];
            A2 o0, o1;
            o0.x = m0r * x.x - m0i * x.y + m1r * y.x - m1i * y.y;
            o0.y = m0r * x.y + m0i * x.x + m1r * y.y + m1i * y.x;
            o1.x = m2r * x.x - m2i * x.y + m3r * y.x - m3i * y.y;
            o1.y = m2r * x.y + m2i * x.x + m3r * y.y + m3i * y.x;
            sm[i0] = o0;
            sm[i1] = o1;
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x) __stcg(state + i, sm[i]);
}

template <typename Real, int R, int W>
__global__ void __launch_bounds__(32 << W) __maxnreg__((pass_max_regs<Real, R>()))
    batch_kernel(const BatchTask *__restrict__ tasks, int ntasks, long long total_items,
                 unsigned long long *next_item, unsigned int *done, int *error) {
    using A2 = typename V2<Real>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    A2 *sm = reinterpret_cast<A2 *>(smem_raw);
    __shared__ long long s_item;
    __shared__ int s_task;
    __shared__ int s_skip;
    // the item's pass arguments, copied once per item into shared memory (the
    // tile code reads them many times; chained kernel, kernels.cu)
    __shared__ __align__(16) PassArgs s_pa;
    for (;;) {
        if (threadIdx.x == 0) {
            const long long it = (long long)atomicAdd(next_item, 1ull);
            s_item = it;
            s_skip = 0;
            if (it < total_items) {
                int lo = 0, hi = ntasks - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (tasks[mid].tile_begin <= it) lo = mid;
                    else hi = mid - 1;
                }
                s_task = lo;
                const int dep = tasks[lo].dep;
                if (dep >= 0) {
                    const unsigned int need = tasks[lo].dep_need;
                    const unsigned long long limit = tasks[lo].wait_ns;
                    const unsigned long long t0 = global_ns();
                    while (ld_acquire(&done[dep]) < need) {
                        if (global_ns() - t0 > limit) {
                            atomicExch(error, 1);
                            s_skip = 1;
                            break;
                        }
                        __nanosleep(128);
                    }
                }
            }
        }
        __syncthreads();
        const long long it = s_item;
        if (it >= total_items) break;
        const BatchTask &t = tasks[s_task];
        if (!s_skip) {
            if (t.small) {
                small_task<Real>(reinterpret_cast<A2 *>(t.state), t.n,
                                 reinterpret_cast<const SmallOp<Real> *>(t.small_ops), t.n_small_ops, sm);
            } else {
                const uint32_t *src = reinterpret_cast<const uint32_t *>(&t.pa);
                uint32_t *dst = reinterpret_cast<uint32_t *>(&s_pa);
                for (int w = threadIdx.x; w < (int)(sizeof(PassArgs) / 4); w += blockDim.x) dst[w] = __ldg(src + w);
                __syncthreads();
                run_tile<Real, R, W>(reinterpret_cast<A2 *>(t.state), s_pa, (uint64_t)(it - t.tile_begin), sm);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(&done[s_task], 1u);
        }
    }
}

template <typename Real>
__global__ void batch_init_kernel(const long long *offsets, const long long *init_index, int njobs,
                                  typename V2<Real>::T *arena) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < njobs) {
        typename V2<Real>::T one;
        one.x = 1;
        one.y = 0;
        arena[offsets[j] + init_index[j]] = one;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

struct BatchJob {
    std::vector<Op> ops;
    int n = 0;
    long long init_index = 0;
    long long offset = 0;   // amplitudes into the arena
    std::unique_ptr<Plan> plan;
};

struct Batch {
    int precision = HGM_F64;
    int warp_bits = 2;
    int low_bits = -1;      // the planner's default when negative
    std::vector<BatchJob> jobs;
    bool finalized = false;
    std::vector<BatchTask> tasks;
    long long total_items = 0;
    size_t arena_bytes = 0;
    void *arena = nullptr;
    BatchTask *d_tasks = nullptr;
    unsigned long long *d_next = nullptr;
    unsigned int *d_done = nullptr;
    int *d_error = nullptr;
    long long *d_offsets = nullptr, *d_init = nullptr;
    int grid = 0;
    int smem = 0;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t stream = nullptr;
    std::vector<State> views;
    ~Batch() { release(); }
    // Drops everything finalize built (plans, arena, tables, graph); the
    // circuits stay, so the batch can be finalized again with other settings.
    void release() {
        if (graph || arena) cudaDeviceSynchronize();  // a replay may still be running
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        for (void *p : {(void *)arena, (void *)d_tasks, (void *)d_next, (void *)d_done, (void *)d_error,
                        (void *)d_offsets, (void *)d_init})
            if (p) cudaFree(p);
        arena = nullptr;
        d_tasks = nullptr;
        d_next = nullptr;
        d_done = nullptr;
        d_error = nullptr;
        d_offsets = d_init = nullptr;
        for (BatchJob &j : jobs) j.plan.reset();
        tasks.clear();
        views.clear();
        total_items = 0;
        arena_bytes = 0;
        finalized = false;
    }
};

namespace {

template <typename Real, int R, int W>
int batch_setup(Batch *b) {
    const int smem = tile_smem_elems<R, W>() * (int)sizeof(typename V2<Real>::T);
    cudaError_t e = cudaFuncSetAttribute(batch_kernel<Real, R, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return fail(HGM_ERR_CUDA, "batch kernel attribute: %s", cudaGetErrorString(e));
    int per_sm = 0, dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<Real, R, W>, 32 << W, smem);
    if (e != cudaSuccess || per_sm < 1) return fail(HGM_ERR_CUDA, "batch kernel occupancy: %s", cudaGetErrorString(e));
    b->grid = sms * per_sm;
    b->smem = smem;
    return HGM_OK;
}

template <typename Real, int R, int W>
void batch_launch(Batch *b, cudaStream_t st) {
    batch_kernel<Real, R, W><<<b->grid, 32 << W, b->smem, st>>>(b->d_tasks, (int)b->tasks.size(), b->total_items,
                                                                 b->d_next, b->d_done, b->d_error);
}

template <typename Real>
int batch_dispatch(Batch *b, bool setup, cudaStream_t st) {
    constexpr int R = sizeof(Real) == 8 ? HGM_F64_REG_BITS : HGM_F32_REG_BITS;
    switch (b->warp_bits) {
        case 0: return setup ? batch_setup<Real, R, 0>(b) : (batch_launch<Real, R, 0>(b, st), HGM_OK);
        case 1: return setup ? batch_setup<Real, R, 1>(b) : (batch_launch<Real, R, 1>(b, st), HGM_OK);
        case 2: return setup ? batch_setup<Real, R, 2>(b) : (batch_launch<Real, R, 2>(b, st), HGM_OK);
        default: return setup ? batch_setup<Real, R, 3>(b) : (batch_launch<Real, R, 3>(b, st), HGM_OK);
    }
}

int cuda_err(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return HGM_OK;
    return fail(e == cudaErrorMemoryAllocation ? HGM_ERR_NOMEM : HGM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int batch_finalize(Batch *b) {
    if (b->finalized) return HGM_OK;
    if (b->jobs.empty()) return fail(HGM_ERR_INVALID, "empty batch");
    const int R = reg_bits_for(b->precision);
    const int K = 5 + R + b->warp_bits;
    const size_t amp = b->precision == HGM_F64 ? 16 : 8;
    // plans and arena layout
    long long off = 0;
    for (BatchJob &j : b->jobs) {
        hgm_plan_opts o;
        hgm_plan_default_opts(&o, b->precision);
        o.renorm_every = 0;
        o.chained = 0;  // the batch kernel runs the passes itself
        o.warp_bits = b->warp_bits;
        o.low_bits = b->low_bits;
        o.reg_bits = R;  // the batch kernel's tile (compile-time R)
        j.plan.reset(new Plan());
        // a state smaller than one tile runs whole in one CTA's shared memory
        int rc = build_plan(j.ops, j.n, o, j.plan.get(), j.n < K);
        if (rc) return rc;
        rc = upload_plan(j.plan.get());
        if (rc) return rc;
        j.offset = off;
        off += 1ll << j.n;
    }
    b->arena_bytes = (size_t)off * amp;
    int rc = cuda_err(cudaMalloc(&b->arena, b->arena_bytes), "batch arena");
    if (rc) return rc;
    // tasks, wave by wave
    std::vector<std::vector<int>> task_of(b->jobs.size());
    size_t max_passes = 0;
    for (BatchJob &j : b->jobs) max_passes = std::max(max_passes, j.plan->small ? (size_t)1 : j.plan->passes.size());
    for (size_t wave = 0; wave < max_passes; wave++) {
        for (size_t ji = 0; ji < b->jobs.size(); ji++) {
            BatchJob &j = b->jobs[ji];
            BatchTask t;
            memset(&t, 0, sizeof t);
            t.state = (char *)b->arena + j.offset * amp;
            t.n = j.n;
            t.dep = wave ? task_of[ji].back() : -1;
            if (j.plan->small) {
                if (wave) continue;
                t.small = 1;
                t.ntiles = 1;
                t.small_ops = j.plan->d_ops;
                t.n_small_ops = j.plan->n_small_ops;
                if (t.n_small_ops == 0) {
                    t.small_ops = nullptr;
                }
            } else {
                if (wave >= j.plan->passes.size()) continue;
                t.pa = j.plan->passes[wave];
                t.pa.flags = 0;
                t.ntiles = 1 << (j.n - t.pa.k);
            }
            t.dep_need = t.dep >= 0 ? (uint32_t)b->tasks[t.dep].ntiles : 0u;
            t.wait_ns = BATCH_WAIT_LIMIT_NS;
            t.tile_begin = b->total_items;
            b->total_items += t.ntiles;
            task_of[ji].push_back((int)b->tasks.size());
            b->tasks.push_back(t);
        }
    }
    // device copies
    const size_t tb = b->tasks.size() * sizeof(BatchTask);
    std::vector<long long> offs, inits;
    for (BatchJob &j : b->jobs) {
        offs.push_back(j.offset);
        inits.push_back(j.init_index);
    }
    if ((rc = cuda_err(cudaMalloc(&b->d_tasks, tb), "batch tasks")) ||
        (rc = cuda_err(cudaMemcpy(b->d_tasks, b->tasks.data(), tb, cudaMemcpyHostToDevice), "batch tasks copy")) ||
        (rc = cuda_err(cudaMalloc(&b->d_next, sizeof(unsigned long long)), "batch counter")) ||
        (rc = cuda_err(cudaMalloc(&b->d_done, b->tasks.size() * sizeof(unsigned int)), "batch done")) ||
        (rc = cuda_err(cudaMalloc(&b->d_error, sizeof(int)), "batch error")) ||
        (rc = cuda_err(cudaMalloc(&b->d_offsets, offs.size() * sizeof(long long)), "batch offsets")) ||
        (rc = cuda_err(cudaMalloc(&b->d_init, inits.size() * sizeof(long long)), "batch inits")) ||
        (rc = cuda_err(cudaMemcpy(b->d_offsets, offs.data(), offs.size() * 8, cudaMemcpyHostToDevice), "offsets")) ||
        (rc = cuda_err(cudaMemcpy(b->d_init, inits.data(), inits.size() * 8, cudaMemcpyHostToDevice), "inits")))
        return rc;
    rc = b->precision == HGM_F64 ? batch_dispatch<double>(b, true, nullptr) : batch_dispatch<float>(b, true, nullptr);
    if (rc) return rc;
    // capture: reset counters and states, run the persistent kernel
    b->stream = (cudaStream_t)default_stream();
    cudaStream_t cap;
    if ((rc = cuda_err(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "capture stream"))) return rc;
    cudaGraph_t g;
    cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    cudaMemsetAsync(b->d_next, 0, sizeof(unsigned long long), cap);
    cudaMemsetAsync(b->d_done, 0, b->tasks.size() * sizeof(unsigned int), cap);
    cudaMemsetAsync(b->d_error, 0, sizeof(int), cap);
    cudaMemsetAsync(b->arena, 0, b->arena_bytes, cap);
    const int nj = (int)b->jobs.size();
    if (b->precision == HGM_F64)
        batch_init_kernel<double><<<(nj + 255) / 256, 256, 0, cap>>>(b->d_offsets, b->d_init, nj, (double2 *)b->arena);
    else
        batch_init_kernel<float><<<(nj + 255) / 256, 256, 0, cap>>>(b->d_offsets, b->d_init, nj, (float2 *)b->arena);
    if (b->precision == HGM_F64) batch_dispatch<double>(b, false, cap);
    else batch_dispatch<float>(b, false, cap);
    cudaError_t e = cudaStreamEndCapture(cap, &g);
    cudaStreamDestroy(cap);
    if ((rc = cuda_err(e, "batch graph capture"))) return rc;
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if ((rc = cuda_err(e, "batch graph instantiate"))) return rc;
    b->views.resize(b->jobs.size());
    for (size_t ji = 0; ji < b->jobs.size(); ji++) {
        b->views[ji].qubits = b->jobs[ji].n;
        b->views[ji].precision = b->precision;
        b->views[ji].d = (char *)b->arena + b->jobs[ji].offset * amp;
        b->views[ji].owned = false;
    }
    b->finalized = true;
    return HGM_OK;
}

}  // namespace
}  // namespace hgm

using namespace hgm;

extern "C" {

int hgm_batch_create(int precision, int warp_bits, hgm_batch **out) {
    if (!out) return fail(HGM_ERR_INVALID, "null output");
    if (precision != HGM_F64 && precision != HGM_F32) return fail(HGM_ERR_INVALID, "bad precision");
    if (!default_stream()) return HGM_ERR_CUDA;
    Batch *b = new Batch();
    b->precision = precision;
    b->warp_bits = warp_bits < 0 ? 2 : std::min(warp_bits, 3);
    *out = reinterpret_cast<hgm_batch *>(b);
    return HGM_OK;
}

void hgm_batch_free(hgm_batch *b) { delete reinterpret_cast<Batch *>(b); }

int hgm_batch_add(hgm_batch *bb, const hgm_circuit *c, int qubits, int64_t init_index, int *job) {
    Batch *b = reinterpret_cast<Batch *>(bb);
    if (!b || !c) return fail(HGM_ERR_INVALID, "null argument");
    if (b->finalized) return fail(HGM_ERR_INVALID, "batch already finalized");
    if (qubits < 1 || qubits > 30) return fail(HGM_ERR_UNSUPPORTED, "batched circuits take 1..30 qubits");
    if (init_index < 0 || init_index >= (1ll << qubits)) return fail(HGM_ERR_INVALID, "initial index outside state");
    BatchJob j;
    j.ops = reinterpret_cast<const Circuit *>(c)->ops;
    j.n = qubits;
    j.init_index = init_index;
    b->jobs.push_back(std::move(j));
    if (job) *job = (int)b->jobs.size() - 1;
    return HGM_OK;
}

int hgm_batch_finalize(hgm_batch *b) {
    if (!b) return fail(HGM_ERR_INVALID, "null batch");
    return batch_finalize(reinterpret_cast<Batch *>(b));
}

int hgm_batch_run(hgm_batch *bb, void *stream) {
    Batch *b = reinterpret_cast<Batch *>(bb);
    if (!b) return fail(HGM_ERR_INVALID, "null batch");
    int rc = batch_finalize(b);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
    cudaError_t e = cudaGraphLaunch(b->graph, st);
    count_launch(2);
    return cuda_err(e, "batch graph launch");
}

int hgm_batch_autotune(hgm_batch *bb, void *stream, int *warp_bits, int *low_bits, double *ms) {
    Batch *b = reinterpret_cast<Batch *>(bb);
    if (!b) return fail(HGM_ERR_INVALID, "null batch");
    if (b->jobs.empty()) return fail(HGM_ERR_INVALID, "empty batch");
    cudaStream_t st = stream ? (cudaStream_t)stream : (cudaStream_t)default_stream();
    // earlier runs of this batch must be done before its buffers are dropped
    if (b->stream) cudaStreamSynchronize(b->stream);
    cudaStreamSynchronize(st);
    cudaEvent_t e0, e1;
    int rc;
    if ((rc = cuda_err(cudaEventCreate(&e0), "autotune event")) || (rc = cuda_err(cudaEventCreate(&e1), "autotune event")))
        return rc;
    // tile size (warps per CTA) x always-resident low index bits: the two
    // settings that decide a plan's pass count and its tile work
    int best_w = -1, best_l = -1;
    float best = 0.f;
    const int lows[3] = {3, 4, 5};
    for (int w = 0; w <= 3 && !rc; w++) {
        for (int li = 0; li < 3 && !rc; li++) {
            b->release();
            b->warp_bits = w;
            b->low_bits = lows[li];
            if ((rc = batch_finalize(b))) break;
            cudaGraphLaunch(b->graph, st);  // warm-up
            cudaEventRecord(e0, st);
            for (int k = 0; k < 2; k++) cudaGraphLaunch(b->graph, st);
            cudaEventRecord(e1, st);
            if ((rc = cuda_err(cudaEventSynchronize(e1), "autotune run"))) break;
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            t *= 0.5f;
            if (best_w < 0 || t < best) {
                best = t;
                best_w = w;
                best_l = lows[li];
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    b->release();
    b->warp_bits = best_w;
    b->low_bits = best_l;
    if ((rc = batch_finalize(b))) return rc;
    if (warp_bits) *warp_bits = best_w;
    if (low_bits) *low_bits = best_l;
    if (ms) *ms = best;
    return HGM_OK;
}

int hgm_batch_set_inputs(hgm_batch *bb, const int64_t *init_index, void *stream) {
    Batch *b = reinterpret_cast<Batch *>(bb);
    if (!b || !init_index) return fail(HGM_ERR_INVALID, "null argument");
    int rc = batch_finalize(b);
    if (rc) return rc;
    for (size_t j = 0; j < b->jobs.size(); j++)
        if (init_index[j] < 0 || init_index[j] >= (1ll << b->jobs[j].n))
            return fail(HGM_ERR_INVALID, "job %zu: initial index outside its state", j);
    for (size_t j = 0; j < b->jobs.size(); j++) b->jobs[j].init_index = init_index[j];
    cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
    return cuda_err(cudaMemcpyAsync(b->d_init, init_index, b->jobs.size() * sizeof(long long), cudaMemcpyHostToDevice, st),
                    "batch inputs");
}

int hgm_batch_download(hgm_batch *bb, void *host, int64_t bytes, void *stream) {
    Batch *b = reinterpret_cast<Batch *>(bb);
    if (!b || !host) return fail(HGM_ERR_INVALID, "null argument");
    if (!b->finalized) return fail(HGM_ERR_INVALID, "batch not finalized");
    if (bytes != (int64_t)b->arena_bytes)
        return fail(HGM_ERR_INVALID, "host buffer of %lld bytes for an arena of %lld", (long long)bytes,
                    (long long)b->arena_bytes);
    cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
    return cuda_err(cudaMemcpyAsync(host, b->arena, b->arena_bytes, cudaMemcpyDeviceToHost, st), "batch download");
}

int hgm_batch_check(hgm_batch *bb) {
    Batch *b = reinterpret_cast<Batch *>(bb);
    if (!b || !b->finalized) return fail(HGM_ERR_INVALID, "batch not run");
    int err = 0;
    cudaError_t e = cudaMemcpy(&err, b->d_error, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_err(e, "batch error flag");
    return err ? fail(HGM_ERR_TIMEOUT, "a batched tile gave up waiting for its previous pass") : HGM_OK;
}

int hgm_batch_inject_stall(hgm_batch *bb, int task, int64_t wait_ns) {
    Batch *b = reinterpret_cast<Batch *>(bb);
    if (!b || !b->finalized) return fail(HGM_ERR_INVALID, "batch not finalized");
    if (task >= (int)b->tasks.size()) return fail(HGM_ERR_INVALID, "no task %d", task);
    if (task >= 0 && b->tasks[task].dep < 0) return fail(HGM_ERR_INVALID, "task %d has no dependency", task);
    if (task >= 0 && wait_ns <= 0) return fail(HGM_ERR_INVALID, "wait limit must be positive");
    for (size_t k = 0; k < b->tasks.size(); k++) {
        BatchTask &t = b->tasks[k];
        t.dep_need = t.dep >= 0 ? (uint32_t)b->tasks[t.dep].ntiles : 0u;
        t.wait_ns = task >= 0 ? (unsigned long long)wait_ns : BATCH_WAIT_LIMIT_NS;
    }
    if (task >= 0) b->tasks[task].dep_need += 1;  // one completion more than the dependency has tiles
    // earlier replays read the table: let them finish before it changes
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_tasks, b->tasks.data(), b->tasks.size() * sizeof(BatchTask), cudaMemcpyHostToDevice);
    return cuda_err(e, "batch task table");
}

int hgm_batch_size(const hgm_batch *bb, int *jobs, int64_t *tasks, int64_t *items, int64_t *arena_bytes,
                   int64_t *pass_bytes) {
    const Batch *b = reinterpret_cast<const Batch *>(bb);
    if (!b) return fail(HGM_ERR_INVALID, "null batch");
    if (jobs) *jobs = (int)b->jobs.size();
    if (tasks) *tasks = (int64_t)b->tasks.size();
    if (items) *items = b->total_items;
    if (arena_bytes) *arena_bytes = (int64_t)b->arena_bytes;
    if (pass_bytes) {  // one read and one write of a state per pass (per shared-memory task)
        const int64_t amp = b->precision == HGM_F64 ? 16 : 8;
        int64_t t = 0;
        for (const BatchTask &k : b->tasks) t += 2 * amp * (int64_t(1) << k.n);
        *pass_bytes = t;
    }
    return HGM_OK;
}

hgm_state *hgm_batch_state(hgm_batch *bb, int job) {
    Batch *b = reinterpret_cast<Batch *>(bb);
    if (!b || !b->finalized || job < 0 || job >= (int)b->jobs.size()) {
        fail(HGM_ERR_INVALID, "no such batched job");
        return nullptr;
    }
    return reinterpret_cast<hgm_state *>(&b->views[job]);
}

}  // extern "C"
