// Kernels and launchers of the state-vector engine (sm_100a).
//
//   pass_kernel<Real, W>   one state pass of a plan (kernels.cuh: run_tile)
//   small_kernel<Real>     states of < 10 qubits: whole state in one CTA's
//                          shared memory, gates applied one by one
//   reduce_*               FP64 reductions (norm, bit probability, inner
//                          product, max |difference|) with a fixed grid and a
//                          fixed combine order, so a result does not depend
//                          on what else runs on the device
//   collapse / scale / set_basis / marginal argmax
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <mutex>

#include "kernels.cuh"

namespace hgm {

// ---------------------------------------------------------------------------
// context: one library stream, a small scratch area for reductions
// ---------------------------------------------------------------------------

namespace {
constexpr int RED_BLOCKS = REDUCE_SCRATCH_BLOCKS;   // 8 x 148 SMs
constexpr int RED_THREADS = 256;

struct Ctx {
    int device = -1;
    cudaStream_t stream = nullptr;
    double *partials = nullptr;    // RED_BLOCKS * 2 doubles
    long long *partial_idx = nullptr;
    double *result = nullptr;      // 4 doubles (device)
    double *host_result = nullptr; // 4 doubles (pinned)
    cudaEvent_t t0 = nullptr, t1 = nullptr;
};
Ctx g_ctx;
std::mutex g_ctx_mu;
std::atomic<long long> g_launches{0};
}  // namespace

void count_launch(int n) { g_launches += n; }

static int ensure_ctx() {
    if (g_ctx.stream) return HGM_OK;
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    if (g_ctx.stream) return HGM_OK;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(HGM_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    g_ctx.device = dev;
    cudaStream_t s;
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(HGM_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    if ((e = cudaMalloc(&g_ctx.partials, RED_BLOCKS * 2 * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&g_ctx.partial_idx, RED_BLOCKS * sizeof(long long))) != cudaSuccess ||
        (e = cudaMalloc(&g_ctx.result, 4 * sizeof(double))) != cudaSuccess ||
        (e = cudaMallocHost(&g_ctx.host_result, 4 * sizeof(double))) != cudaSuccess ||
        (e = cudaEventCreate(&g_ctx.t0)) != cudaSuccess || (e = cudaEventCreate(&g_ctx.t1)) != cudaSuccess)
        return fail(HGM_ERR_CUDA, "context setup: %s", cudaGetErrorString(e));
    g_ctx.stream = s;
    return HGM_OK;
}

void *default_stream() {
    if (ensure_ctx() != HGM_OK) return nullptr;
    return g_ctx.stream;
}

static inline cudaStream_t pick(void *stream) {
    return stream ? (cudaStream_t)stream : (cudaStream_t)default_stream();
}

static inline int check(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(HGM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return HGM_OK;
}

// ---------------------------------------------------------------------------
// pass kernels
// ---------------------------------------------------------------------------

template <typename Real, int R, int W, bool LEAN>
__global__ void __launch_bounds__(32 << W) __maxnreg__((pass_max_regs<Real, R>()))
    pass_kernel(typename V2<Real>::T *__restrict__ state, const PassArgs pa) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    run_tile<Real, R, W, LEAN>(state, pa, blockIdx.x, reinterpret_cast<typename V2<Real>::T *>(smem_raw));
}

template <typename Real>
__global__ void __launch_bounds__(256) small_kernel(typename V2<Real>::T *__restrict__ state, int n,
                                                    const SmallOp<Real> *__restrict__ ops, long long n_ops,
                                                    int iterations) {
    using A2 = typename V2<Real>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    A2 *sm = reinterpret_cast<A2 *>(smem_raw);
    const int N = 1 << n, half = N >> 1;
    for (int i = threadIdx.x; i < N; i += blockDim.x) sm[i] = state[i];
    __syncthreads();
    for (int it = 0; it < iterations; it++) {
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
    }
    for (int i = threadIdx.x; i < N; i += blockDim.x) state[i] = sm[i];
}

template <typename Real, int R, int W, bool LEAN>
static int setup_pass_kernel() {
    static bool done = false;
    if (done) return HGM_OK;
    const int smem = tile_smem_elems<R, W>() * (int)sizeof(typename V2<Real>::T);
    cudaError_t e =
        cudaFuncSetAttribute(pass_kernel<Real, R, W, LEAN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess && HGM_SMEM_CARVEOUT >= 0)
        e = cudaFuncSetAttribute(pass_kernel<Real, R, W, LEAN>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 HGM_SMEM_CARVEOUT);
    if (e != cudaSuccess) return fail(HGM_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    done = true;
    return HGM_OK;
}

template <typename Real, int R, int W, bool LEAN>
static int launch_pass(void *state, const PassArgs &pa, cudaStream_t st) {
    using A2 = typename V2<Real>::T;
    int rc = setup_pass_kernel<Real, R, W, LEAN>();
    if (rc) return rc;
    const uint64_t tiles = 1ull << (pa.n - pa.k);
    const int smem = tile_smem_elems<R, W>() * (int)sizeof(A2);
    pass_kernel<Real, R, W, LEAN><<<(unsigned)tiles, 32 << W, smem, st>>>(reinterpret_cast<A2 *>(state), pa);
    count_launch();
    return HGM_OK;
}

// FP64 tiles hold 16 amplitudes a thread (R = 4), FP32 tiles 32 (R = 5) or,
// on request, 16 (plan_reg_bits).
template <typename Real, int R, bool LEAN>
static int launch_pass_w(int W, void *state, const PassArgs &pa, cudaStream_t st) {
    switch (W) {
        case 0: return launch_pass<Real, R, 0, LEAN>(state, pa, st);
        case 1: return launch_pass<Real, R, 1, LEAN>(state, pa, st);
        case 2: return launch_pass<Real, R, 2, LEAN>(state, pa, st);
        default: return launch_pass<Real, R, 3, LEAN>(state, pa, st);
    }
}
template <typename Real, int R>
static int launch_pass_lw(bool lean, int W, void *state, const PassArgs &pa, cudaStream_t st) {
    return lean ? launch_pass_w<Real, R, true>(W, state, pa, st) : launch_pass_w<Real, R, false>(W, state, pa, st);
}

template <typename Real>
static int launch_small(State *s, const Plan *p, int iterations, cudaStream_t st) {
    const int smem = (1 << s->qubits) * (int)sizeof(typename V2<Real>::T);
    small_kernel<Real><<<1, 256, smem, st>>>(reinterpret_cast<typename V2<Real>::T *>(s->d), s->qubits,
                                             reinterpret_cast<const SmallOp<Real> *>(p->d_ops), p->n_small_ops,
                                             iterations);
    count_launch();
    return check("small_kernel launch");
}

int launch_plan_steps(State *s, const Plan *p, int iterations, PlanCursor *c, int64_t max_launches, void *stream) {
    if (s->qubits != p->qubits) return fail(HGM_ERR_INVALID, "plan is for %d qubits, state has %d", p->qubits, s->qubits);
    if (s->precision != p->precision) return fail(HGM_ERR_INVALID, "plan and state precision differ");
    // every device pointer a launch passes must exist: an op list that was
    // never uploaded is refused here, not read through a null pointer
    if ((!p->ops_bytes.empty() && !p->d_ops) || (!p->phases.empty() && !p->d_phases) ||
        (!p->layouts.empty() && !p->d_layouts) ||
        (p->renorm_every > 0 && !p->small && !p->d_norm))
        return fail(HGM_ERR_INVALID, "plan used before upload_plan");
    cudaStream_t st = pick(stream);
    if (!st) return HGM_ERR_CUDA;
    if (p->small) {
        if (c->next > 0 || max_launches < 1) return HGM_OK;
        c->next = 1;
        return p->n_small_ops ? (p->precision == HGM_F64 ? launch_small<double>(s, p, iterations, st)
                                                         : launch_small<float>(s, p, iterations, st))
                              : HGM_OK;
    }
    const int64_t np = (int64_t)p->passes.size();
    const int R = p->renorm_every;
    const int64_t total = np * iterations;
    for (int64_t k = 0; k < max_launches && c->next < total; k++, c->next++) {
        const int64_t g = c->next;
        PassArgs pa = p->passes[g % np];
        pa.flags = 0;
        if (c->scale_next) {
            pa.flags |= PASS_SCALE;
            pa.scale_in = p->d_norm + c->scale_slot;
            c->scale_next = false;
        }
        if (R > 0 && ((g + 1) % R == 0) && g + 1 < total) {
            pa.flags |= PASS_NORM;
            pa.norm_out = p->d_norm + c->slot;
            cudaMemsetAsync(pa.norm_out, 0, sizeof(double), st);
            c->scale_next = true;
            c->scale_slot = c->slot;
            c->slot = (c->slot + 1) % 64;
        }
        int rc = p->precision == HGM_F64
                     ? launch_pass_lw<double, HGM_F64_REG_BITS>(p->lean, p->warp_bits, s->d, pa, st)
                 : p->reg_bits == 4 ? launch_pass_lw<float, 4>(p->lean, p->warp_bits, s->d, pa, st)
                                    : launch_pass_lw<float, HGM_F32_REG_BITS>(p->lean, p->warp_bits, s->d, pa, st);
        if (rc) return rc;
    }
    return check("pass_kernel launch");
}

int64_t plan_launches(const Plan *p, int iterations) {
    return p->small ? 1 : (int64_t)p->passes.size() * iterations;
}

// ---------------------------------------------------------------------------
// chained passes: every pass of a small state in one persistent launch
// ---------------------------------------------------------------------------
// A state that fits in L2 moves through a pass in a few microseconds, so
// launching one kernel per pass leaves it bound by launch latency and the
// tail of each launch.  The chained kernel runs the whole pass sequence in
// one launch.  Its CTAs claim work items (pass g, tile t) in sequence order
// from a counter, and the CTA that claimed an item of pass g waits until
// every item of passes 0..g-1 is done (a second counter) before it loads.
// An item only waits for items claimed before it, and a claimed item is held
// by a running CTA, so the sequence always progresses whether or not all of
// the grid is resident.  The wait is bounded (2 s of %globaltimer); a CTA
// that gives up sets the error word and skips its tile.
//
// Scratch (Plan::d_chain): claim counter, done counter, error word, one
// unused word, then CHAIN_NORM_SLOTS FP64 norm slots used in turn, so that a
// sequence of any length (many iterations of a short FP32 plan) runs chained.
// Renormalisation k accumulates into slot k % CHAIN_NORM_SLOTS during pass
// (k + 1) * renorm - 1 and is read during the next pass; tile 0 of the pass
// before an accumulating pass zeroes its slot before counting itself done, so
// the zero is seen by every tile of that pass (they wait for the count) and
// comes after the slot's previous reads (three slots: CHAIN_NORM_SLOTS *
// renorm > 2 passes apart).
constexpr unsigned long long CHAIN_WAIT_LIMIT_NS = 2000000000ull;
constexpr int CHAIN_NORM_SLOTS = 3;

__device__ __forceinline__ unsigned long long chain_now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

template <typename Real, int R, int W, bool LEAN>
__global__ void __launch_bounds__(32 << W) __maxnreg__((pass_max_regs<Real, R>()))
    chain_kernel(typename V2<Real>::T *__restrict__ state, const PassArgs *__restrict__ passes, int npasses,
                 int tile_bits, long long total, int renorm, unsigned long long *ctr, double *norms) {
    using A2 = typename V2<Real>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    A2 *sm = reinterpret_cast<A2 *>(smem_raw);
    __shared__ long long s_item;
    __shared__ int s_skip;
    // the item's pass arguments, copied once per item: the tile code reads
    // them many times (the tile-bit map byte by byte), from shared memory
    // rather than through L1
    __shared__ __align__(16) PassArgs s_pa;
    static_assert(sizeof(PassArgs) % 4 == 0, "PassArgs copies as words");
    const long long seq = total >> tile_bits;  // passes in the sequence
    for (;;) {
        if (threadIdx.x == 0) {
            const long long it = (long long)atomicAdd(&ctr[0], 1ull);
            s_item = it;
            s_skip = 0;
            if (it < total) {
                const unsigned long long need = (unsigned long long)((it >> tile_bits) << tile_bits);
                const unsigned long long t0 = chain_now_ns();
                while (ld_acquire_u64(&ctr[1]) < need) {
                    if (chain_now_ns() - t0 > CHAIN_WAIT_LIMIT_NS) {
                        atomicExch(&ctr[2], 1ull);
                        s_skip = 1;
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
        __syncthreads();
        const long long it = s_item;
        if (it >= total) break;
        if (!s_skip) {
            const long long g = it >> tile_bits;
            int32_t flags = 0;
            double *norm_out = nullptr;
            const double *scale_in = nullptr;
            if (renorm > 0) {
                // the plain launcher's schedule: a norm on every renorm-th
                // pass but the last, a rescale on the pass after it
                if ((g + 1) % renorm == 0 && g + 1 < seq) {
                    flags |= PASS_NORM;
                    norm_out = norms + ((g + 1) / renorm - 1) % CHAIN_NORM_SLOTS;
                }
                if (g > 0 && g % renorm == 0) {
                    flags |= PASS_SCALE;
                    scale_in = norms + (g / renorm - 1) % CHAIN_NORM_SLOTS;
                }
            }
            {
                const uint32_t *src = reinterpret_cast<const uint32_t *>(passes + g % npasses);
                uint32_t *dst = reinterpret_cast<uint32_t *>(&s_pa);
                for (int w = threadIdx.x; w < (int)(sizeof(PassArgs) / 4); w += blockDim.x) dst[w] = __ldg(src + w);
            }
            __syncthreads();
            run_tile<Real, R, W, LEAN>(state, s_pa, (uint64_t)(it & ((1ll << tile_bits) - 1)), sm, flags, norm_out,
                                       scale_in);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const long long g = it >> tile_bits;
            // the next pass accumulates a norm: zero its slot first
            if (renorm > 0 && (it & ((1ll << tile_bits) - 1)) == 0 && (g + 2) % renorm == 0 && g + 2 < seq)
                norms[((g + 2) / renorm - 1) % CHAIN_NORM_SLOTS] = 0.0;
            __threadfence();
            atomicAdd(&ctr[1], 1ull);
        }
    }
}

template <typename Real, int R, int W, bool LEAN>
static int launch_chain_rw(State *s, const Plan *p, int iterations, cudaStream_t st) {
    using A2 = typename V2<Real>::T;
    static int grid_cap = 0;
    const int smem = tile_smem_elems<R, W>() * (int)sizeof(A2);
    if (!grid_cap) {
        cudaError_t e = cudaFuncSetAttribute(chain_kernel<Real, R, W, LEAN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        int per_sm = 0, dev = 0, sms = 0;
        if (e == cudaSuccess) e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, chain_kernel<Real, R, W, LEAN>, 32 << W, smem);
        if (e != cudaSuccess || per_sm < 1) return fail(HGM_ERR_CUDA, "chain kernel setup: %s", cudaGetErrorString(e));
        grid_cap = sms * per_sm;
    }
    const int tile_bits = p->qubits - p->passes[0].k;
    const long long total = ((long long)p->passes.size() * iterations) << tile_bits;
    const long long ntiles = 1ll << tile_bits;
    const unsigned grid = (unsigned)(ntiles < grid_cap ? ntiles : grid_cap);
    unsigned long long *ctr = reinterpret_cast<unsigned long long *>(p->d_chain);
    double *norms = reinterpret_cast<double *>(ctr + 4);
    cudaError_t e = cudaMemsetAsync(p->d_chain, 0, p->d_bytes[4], st);
    if (e != cudaSuccess) return fail(HGM_ERR_CUDA, "chain scratch reset: %s", cudaGetErrorString(e));
    chain_kernel<Real, R, W, LEAN><<<grid, 32 << W, smem, st>>>(reinterpret_cast<A2 *>(s->d),
                                                          reinterpret_cast<const PassArgs *>(p->d_chain_passes),
                                                          (int)p->passes.size(), tile_bits, total, p->renorm_every,
                                                          ctr, norms);
    count_launch();
    return check("chain_kernel launch");
}

template <typename Real, int R, bool LEAN>
static int launch_chain_lw(State *s, const Plan *p, int iterations, cudaStream_t st) {
    switch (p->warp_bits) {
        case 0: return launch_chain_rw<Real, R, 0, LEAN>(s, p, iterations, st);
        case 1: return launch_chain_rw<Real, R, 1, LEAN>(s, p, iterations, st);
        case 2: return launch_chain_rw<Real, R, 2, LEAN>(s, p, iterations, st);
        default: return launch_chain_rw<Real, R, 3, LEAN>(s, p, iterations, st);
    }
}
template <typename Real, int R>
static int launch_chain_w(State *s, const Plan *p, int iterations, cudaStream_t st) {
    return p->lean ? launch_chain_lw<Real, R, true>(s, p, iterations, st)
                   : launch_chain_lw<Real, R, false>(s, p, iterations, st);
}

bool chain_eligible(const Plan *p, int iterations) {
    if (p->small || !p->d_chain || p->passes.size() < 2 || iterations < 1) return false;
    const int64_t seq = (int64_t)p->passes.size() * iterations;
    (void)seq;
    return true;
}

int launch_plan_chain(State *s, const Plan *p, int iterations, void *stream) {
    if (s->qubits != p->qubits || s->precision != p->precision)
        return fail(HGM_ERR_INVALID, "plan and state differ in size or precision");
    if (!chain_eligible(p, iterations)) return fail(HGM_ERR_INVALID, "plan not set up for chained passes");
    cudaStream_t st = pick(stream);
    if (!st) return HGM_ERR_CUDA;
    if (p->precision == HGM_F64) return launch_chain_w<double, HGM_F64_REG_BITS>(s, p, iterations, st);
    return p->reg_bits == 4 ? launch_chain_w<float, 4>(s, p, iterations, st)
                            : launch_chain_w<float, HGM_F32_REG_BITS>(s, p, iterations, st);
}

// Error word of the last chained run of `p` (device address, for an
// asynchronous copy after the run).
const void *chain_error_word(const Plan *p) {
    return p->d_chain ? reinterpret_cast<const unsigned long long *>(p->d_chain) + 2 : nullptr;
}

int launch_plan(State *s, const Plan *p, int iterations, void *stream) {
    PlanCursor c;
    return launch_plan_steps(s, p, iterations, &c, plan_launches(p, iterations), stream);
}

// ---------------------------------------------------------------------------
// plan upload
// ---------------------------------------------------------------------------

static cudaError_t plan_alloc(Plan *p, int k, void **out, size_t bytes) {
    p->d_bytes[k] = bytes;
    return p->allocator ? p->allocator->alloc(out, bytes) : cudaMalloc(out, bytes);
}

Plan::~Plan() {
    void *ptrs[6] = {d_ops, d_phases, d_layouts, d_norm, d_chain, d_chain_passes};
    for (int k = 0; k < 6; k++) {
        if (!ptrs[k]) continue;
        if (allocator) allocator->free(ptrs[k], d_bytes[k]);
        else cudaFree(ptrs[k]);
    }
}

int upload_plan(Plan *p) {
    if (p->d_ops || (p->ops_bytes.empty() && p->phases.empty() && !p->renorm_every)) return HGM_OK;
    if (ensure_ctx()) return HGM_ERR_CUDA;
    cudaError_t e;
    if (!p->ops_bytes.empty()) {
        if ((e = plan_alloc(p, 0, &p->d_ops, p->ops_bytes.size())) != cudaSuccess)
            return fail(HGM_ERR_NOMEM, "plan ops: %s", cudaGetErrorString(e));
        if ((e = cudaMemcpy(p->d_ops, p->ops_bytes.data(), p->ops_bytes.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return fail(HGM_ERR_CUDA, "plan ops copy: %s", cudaGetErrorString(e));
    }
    if (!p->phases.empty()) {
        size_t b = p->phases.size() * sizeof(DevPhase);
        if ((e = plan_alloc(p, 1, &p->d_phases, b)) != cudaSuccess) return fail(HGM_ERR_NOMEM, "plan phases: %s", cudaGetErrorString(e));
        if ((e = cudaMemcpy(p->d_phases, p->phases.data(), b, cudaMemcpyHostToDevice)) != cudaSuccess)
            return fail(HGM_ERR_CUDA, "plan phases copy: %s", cudaGetErrorString(e));
    }
    if (!p->layouts.empty()) {
        // per layout: the byte step of each register bit, then each thread's
        // register-0 offset, in the padded transpose buffer (kernels.cuh)
        const int R = p->reg_bits, W = p->warp_bits, nt = 32 << W;
        const uint32_t esz = p->precision == HGM_F64 ? 16 : 8;
        auto pad = [&](uint32_t j) { return (j + (j >> R)) * esz; };
        std::vector<uint32_t> tab(p->layouts.size() * (LAYOUT_HDR + nt), 0u);
        for (size_t l = 0; l < p->layouts.size(); l++) {
            const Lay &lay = p->layouts[l];
            uint32_t *e0 = tab.data() + l * (LAYOUT_HDR + nt);
            for (int q = 0; q < R; q++) e0[q] = pad(1u << lay.pos[5 + W + q]);
            for (int t = 0; t < nt; t++) {
                uint32_t o = 0;
                for (int b = 0; b < 5 + W; b++)
                    if ((t >> b) & 1) o += pad(1u << lay.pos[b]);
                e0[LAYOUT_HDR + t] = o;
            }
        }
        const size_t b = tab.size() * sizeof(uint32_t);
        if ((e = plan_alloc(p, 2, &p->d_layouts, b)) != cudaSuccess)
            return fail(HGM_ERR_NOMEM, "plan layouts: %s", cudaGetErrorString(e));
        if ((e = cudaMemcpy(p->d_layouts, tab.data(), b, cudaMemcpyHostToDevice)) != cudaSuccess)
            return fail(HGM_ERR_CUDA, "plan layouts copy: %s", cudaGetErrorString(e));
    }
    if (p->renorm_every > 0) {
        if ((e = plan_alloc(p, 3, (void **)&p->d_norm, 64 * sizeof(double))) != cudaSuccess)
            return fail(HGM_ERR_NOMEM, "plan norm slots: %s", cudaGetErrorString(e));
    }
    for (PassArgs &pa : p->passes) {
        pa.phases = reinterpret_cast<const DevPhase *>(p->d_phases);
        pa.layouts = reinterpret_cast<const uint32_t *>(p->d_layouts);
        pa.ops = p->d_ops;
    }
    const int64_t state_bytes = (int64_t(1) << p->qubits) * (p->precision == HGM_F64 ? 16 : 8);
    if (p->chained && !p->small && p->passes.size() >= 2 && state_bytes <= CHAIN_MAX_BYTES) {
        // chained execution: the pass records (pointers patched) and the scratch
        p->chain_slots = p->renorm_every > 0 ? CHAIN_NORM_SLOTS : 0;
        const size_t sb = (4 + (size_t)p->chain_slots) * sizeof(double);
        const size_t pb = p->passes.size() * sizeof(PassArgs);
        if ((e = plan_alloc(p, 4, &p->d_chain, sb)) != cudaSuccess)
            return fail(HGM_ERR_NOMEM, "plan chain scratch: %s", cudaGetErrorString(e));
        if ((e = plan_alloc(p, 5, &p->d_chain_passes, pb)) != cudaSuccess)
            return fail(HGM_ERR_NOMEM, "plan chain passes: %s", cudaGetErrorString(e));
        std::vector<PassArgs> dev(p->passes);
        for (PassArgs &pa : dev) {
            pa.flags = 0;
            pa.norm_out = nullptr;
            pa.scale_in = nullptr;
        }
        if ((e = cudaMemcpy(p->d_chain_passes, dev.data(), pb, cudaMemcpyHostToDevice)) != cudaSuccess)
            return fail(HGM_ERR_CUDA, "plan chain passes copy: %s", cudaGetErrorString(e));
    }
    return HGM_OK;
}

// ---------------------------------------------------------------------------
// elementwise kernels
// ---------------------------------------------------------------------------

template <typename Real>
__global__ void set_basis_kernel(typename V2<Real>::T *s, long long N, long long index) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        typename V2<Real>::T v;
        v.x = (i == index) ? (Real)1 : (Real)0;
        v.y = 0;
        s[i] = v;
    }
}

template <typename Real>
__global__ void collapse_kernel(typename V2<Real>::T *s, long long N, int bit, int value, double inv_norm) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        typename V2<Real>::T v = s[i];
        if ((int)((i >> bit) & 1) == value) {
            v.x = (Real)(v.x * inv_norm);
            v.y = (Real)(v.y * inv_norm);
        } else {
            v.x = 0;
            v.y = 0;
        }
        s[i] = v;
    }
}

// DGM::measure(int)'s state update (src/core/dgm_core.cpp:117-122): for every
// pair of indices differing only in `bit`, the amplitude of the measured
// branch, rescaled, goes to the bit-0 index and the bit-1 index is cleared,
// so the measured qubit is left in |0> whichever value was read.  One thread
// per pair: the pair's two amplitudes are read before either is written.
template <typename Real>
__global__ void measure_update_kernel(typename V2<Real>::T *s, long long half, int bit, int value, double inv_norm) {
    const long long low = (1ll << bit) - 1;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < half; p += (long long)gridDim.x * blockDim.x) {
        const long long i0 = ((p & ~low) << 1) | (p & low), i1 = i0 | (1ll << bit);
        typename V2<Real>::T v = s[value ? i1 : i0], z;
        v.x = (Real)(v.x * inv_norm);
        v.y = (Real)(v.y * inv_norm);
        z.x = 0;
        z.y = 0;
        s[i0] = v;
        s[i1] = z;
    }
}

template <typename Real>
__global__ void scale_kernel(typename V2<Real>::T *s, long long N, double f) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        typename V2<Real>::T v = s[i];
        v.x = (Real)(v.x * f);
        v.y = (Real)(v.y * f);
        s[i] = v;
    }
}

static unsigned grid_for(long long N) {
    long long g = (N + 255) / 256;
    return (unsigned)(g < RED_BLOCKS ? (g < 1 ? 1 : g) : RED_BLOCKS);
}

int launch_set_basis(State *s, int64_t index, void *stream) {
    cudaStream_t st = pick(stream);
    if (!st) return HGM_ERR_CUDA;
    long long N = 1ll << s->qubits;
    if (index < 0 || index >= N) return fail(HGM_ERR_INVALID, "basis index %lld outside state", (long long)index);
    if (s->precision == HGM_F64) set_basis_kernel<double><<<grid_for(N), 256, 0, st>>>((double2 *)s->d, N, index);
    else set_basis_kernel<float><<<grid_for(N), 256, 0, st>>>((float2 *)s->d, N, index);
    count_launch();
    return check("set_basis");
}

int collapse(State *s, int bit, int value, double inv_norm, void *stream) {
    cudaStream_t st = pick(stream);
    long long N = 1ll << s->qubits;
    if (s->precision == HGM_F64) collapse_kernel<double><<<grid_for(N), 256, 0, st>>>((double2 *)s->d, N, bit, value, inv_norm);
    else collapse_kernel<float><<<grid_for(N), 256, 0, st>>>((float2 *)s->d, N, bit, value, inv_norm);
    count_launch();
    return check("collapse");
}

int measure_update(State *s, int bit, int value, double inv_norm, void *stream) {
    cudaStream_t st = pick(stream);
    const long long half = 1ll << (s->qubits - 1);
    if (s->precision == HGM_F64)
        measure_update_kernel<double><<<grid_for(half), 256, 0, st>>>((double2 *)s->d, half, bit, value, inv_norm);
    else
        measure_update_kernel<float><<<grid_for(half), 256, 0, st>>>((float2 *)s->d, half, bit, value, inv_norm);
    count_launch();
    return check("measure update");
}

int scale_state(State *s, double f, void *stream) {
    cudaStream_t st = pick(stream);
    long long N = 1ll << s->qubits;
    if (s->precision == HGM_F64) scale_kernel<double><<<grid_for(N), 256, 0, st>>>((double2 *)s->d, N, f);
    else scale_kernel<float><<<grid_for(N), 256, 0, st>>>((float2 *)s->d, N, f);
    count_launch();
    return check("scale");
}

// ---------------------------------------------------------------------------
// FP64 reductions (fixed grid, fixed combine order)
// ---------------------------------------------------------------------------

enum RedMode { RED_NORM = 0, RED_PROB1 = 1, RED_INNER = 2, RED_MAXDIFF = 3 };

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template <typename RA, typename RB, int MODE>
__global__ void __launch_bounds__(RED_THREADS) reduce_kernel(const typename V2<RA>::T *__restrict__ a,
                                                              const typename V2<RB>::T *__restrict__ b, long long N,
                                                              int bit, double *partials) {
    double s0 = 0.0, s1 = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const typename V2<RA>::T x = a[i];
        if (MODE == RED_NORM) {
            s0 += (double)x.x * x.x + (double)x.y * x.y;
        } else if (MODE == RED_PROB1) {
            if ((i >> bit) & 1) s0 += (double)x.x * x.x + (double)x.y * x.y;
        } else if (MODE == RED_INNER) {
            const typename V2<RB>::T y = b[i];
            // conj(x) * y
            s0 += (double)x.x * y.x + (double)x.y * y.y;
            s1 += (double)x.x * y.y - (double)x.y * y.x;
        } else {
            const typename V2<RB>::T y = b[i];
            const double dr = (double)x.x - (double)y.x, di = (double)x.y - (double)y.y;
            s0 = fmax(s0, sqrt(dr * dr + di * di));
        }
    }
    __shared__ double sh[2][RED_THREADS / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (MODE == RED_MAXDIFF) s0 = warp_max(s0);
    else {
        s0 = warp_sum(s0);
        s1 = warp_sum(s1);
    }
    if (lane == 0) {
        sh[0][w] = s0;
        sh[1][w] = s1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int k = 0; k < RED_THREADS / 32; k++) {
            if (MODE == RED_MAXDIFF) t0 = fmax(t0, sh[0][k]);
            else t0 += sh[0][k];
            t1 += sh[1][k];
        }
        partials[2 * blockIdx.x] = t0;
        partials[2 * blockIdx.x + 1] = t1;
    }
}

template <int MODE>
__global__ void reduce_final(const double *partials, int nblocks, double *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int k = 0; k < nblocks; k++) {
            if (MODE == RED_MAXDIFF) t0 = fmax(t0, partials[2 * k]);
            else t0 += partials[2 * k];
            t1 += partials[2 * k + 1];
        }
        out[0] = t0;
        out[1] = t1;
    }
}

template <typename RA, typename RB, int MODE>
static int run_reduce(const void *a, const void *b, int qubits, int bit, double *o0, double *o1, cudaStream_t st) {
    const long long N = 1ll << qubits;
    const unsigned g = grid_for(N);
    reduce_kernel<RA, RB, MODE><<<g, RED_THREADS, 0, st>>>((const typename V2<RA>::T *)a,
                                                           (const typename V2<RB>::T *)b, N, bit, g_ctx.partials);
    reduce_final<MODE><<<1, 32, 0, st>>>(g_ctx.partials, (int)g, g_ctx.result);
    count_launch(2);
    cudaMemcpyAsync(g_ctx.host_result, g_ctx.result, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(HGM_ERR_CUDA, "reduction: %s", cudaGetErrorString(e));
    if (o0) *o0 = g_ctx.host_result[0];
    if (o1) *o1 = g_ctx.host_result[1];
    return HGM_OK;
}

int launch_norm_async(State *s, double *partials, double *out, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    const long long N = 1ll << s->qubits;
    const unsigned g = grid_for(N);
    if (s->precision == HGM_F64)
        reduce_kernel<double, double, RED_NORM><<<g, RED_THREADS, 0, st>>>((const double2 *)s->d, nullptr, N, 0, partials);
    else
        reduce_kernel<float, float, RED_NORM><<<g, RED_THREADS, 0, st>>>((const float2 *)s->d, nullptr, N, 0, partials);
    reduce_final<RED_NORM><<<1, 32, 0, st>>>(partials, (int)g, out);
    count_launch(2);
    return check("norm reduction launch");
}

int reduce_norm(State *s, double *out, void *stream) {
    cudaStream_t st = pick(stream);
    if (!st) return HGM_ERR_CUDA;
    return s->precision == HGM_F64 ? run_reduce<double, double, RED_NORM>(s->d, nullptr, s->qubits, 0, out, nullptr, st)
                                   : run_reduce<float, float, RED_NORM>(s->d, nullptr, s->qubits, 0, out, nullptr, st);
}

int reduce_prob_one(State *s, int bit, double *out, void *stream) {
    cudaStream_t st = pick(stream);
    if (!st) return HGM_ERR_CUDA;
    if (bit < 0 || bit >= s->qubits) return fail(HGM_ERR_INVALID, "bit %d outside state", bit);
    return s->precision == HGM_F64 ? run_reduce<double, double, RED_PROB1>(s->d, nullptr, s->qubits, bit, out, nullptr, st)
                                   : run_reduce<float, float, RED_PROB1>(s->d, nullptr, s->qubits, bit, out, nullptr, st);
}

template <int MODE>
static int two_state(State *a, State *b, double *o0, double *o1, cudaStream_t st) {
    if (a->qubits != b->qubits) return fail(HGM_ERR_INVALID, "states differ in size");
    if (a->precision == HGM_F64 && b->precision == HGM_F64)
        return run_reduce<double, double, MODE>(a->d, b->d, a->qubits, 0, o0, o1, st);
    if (a->precision == HGM_F64) return run_reduce<double, float, MODE>(a->d, b->d, a->qubits, 0, o0, o1, st);
    if (b->precision == HGM_F64) return run_reduce<float, double, MODE>(a->d, b->d, a->qubits, 0, o0, o1, st);
    return run_reduce<float, float, MODE>(a->d, b->d, a->qubits, 0, o0, o1, st);
}

int inner(State *a, State *b, double *re, double *im, void *stream) {
    cudaStream_t st = pick(stream);
    if (!st) return HGM_ERR_CUDA;
    return two_state<RED_INNER>(a, b, re, im, st);
}

int max_abs_diff(State *a, State *b, double *out, void *stream) {
    cudaStream_t st = pick(stream);
    if (!st) return HGM_ERR_CUDA;
    return two_state<RED_MAXDIFF>(a, b, out, nullptr, st);
}

// Marginal argmax: for every value x of the bits in `mask`, p(x) = sum over
// the other bits of |a|^2; returns the x with the largest p (lowest on ties).
// Each thread owns marginal values x and walks the complement bits.
template <typename Real>
__global__ void __launch_bounds__(RED_THREADS) marginal_kernel(const typename V2<Real>::T *__restrict__ s, int n,
                                                                unsigned long long mask, int m, double *pbest,
                                                                long long *ibest) {
    const unsigned long long comp = ~mask & ((n >= 64) ? ~0ull : ((1ull << n) - 1));
    const long long M = 1ll << m, C = 1ll << (n - m);
    double best = -1.0;
    long long besti = 0;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < M; x += (long long)gridDim.x * blockDim.x) {
        // deposit x into mask bits
        unsigned long long base = 0, src = (unsigned long long)x, mm = mask;
        while (mm) {
            int g = __ffsll((long long)mm) - 1;
            mm &= mm - 1;
            base |= (src & 1ull) << g;
            src >>= 1;
        }
        double p = 0.0;
        for (long long c = 0; c < C; c++) {
            unsigned long long idx = base, cs = (unsigned long long)c, cm = comp;
            while (cm) {
                int g = __ffsll((long long)cm) - 1;
                cm &= cm - 1;
                idx |= (cs & 1ull) << g;
                cs >>= 1;
            }
            const typename V2<Real>::T v = s[idx];
            p += (double)v.x * v.x + (double)v.y * v.y;
        }
        if (p > best) {
            best = p;
            besti = x;
        }
    }
    __shared__ double sp[RED_THREADS];
    __shared__ long long si[RED_THREADS];
    sp[threadIdx.x] = best;
    si[threadIdx.x] = besti;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = -1.0;
        long long bi = 0;
        for (int k = 0; k < RED_THREADS; k++)
            if (sp[k] > b || (sp[k] == b && si[k] < bi)) {
                b = sp[k];
                bi = si[k];
            }
        pbest[blockIdx.x] = b;
        ibest[blockIdx.x] = bi;
    }
}

__global__ void marginal_final(const double *pbest, const long long *ibest, int nb, double *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double b = -1.0;
        long long bi = 0;
        for (int k = 0; k < nb; k++)
            if (pbest[k] > b || (pbest[k] == b && ibest[k] < bi)) {
                b = pbest[k];
                bi = ibest[k];
            }
        out[0] = b;
        out[1] = (double)bi;
    }
}

// Marginal argmax for a small mask (2^m <= RED_BLOCKS values): block b
// handles value x = b / nch over the (b % nch)-th chunk of the complement
// indices, its threads striding over the chunk, and writes that chunk's
// probability; marginal_chunks_final sums each value's chunks in order.  With
// the per-value kernel above, a thread would walk all 2^(n-m) complement
// indices of its value alone (minutes for a few-bit mask on a 32-qubit state).
template <typename Real>
__global__ void __launch_bounds__(RED_THREADS) marginal_chunk_kernel(const typename V2<Real>::T *__restrict__ s, int n,
                                                                      unsigned long long mask, int nch,
                                                                      double *partial) {
    const unsigned long long comp = ~mask & ((n >= 64) ? ~0ull : ((1ull << n) - 1));
    const long long C = 1ll << (n - __popcll(mask));
    const long long x = blockIdx.x / nch, chunk = blockIdx.x % nch;
    const long long cs = (C + nch - 1) / nch, c0 = chunk * cs, c1 = c0 + cs < C ? c0 + cs : C;
    unsigned long long base = 0, src = (unsigned long long)x, mm = mask;
    while (mm) {
        const int g = __ffsll((long long)mm) - 1;
        mm &= mm - 1;
        base |= (src & 1ull) << g;
        src >>= 1;
    }
    double p = 0.0;
    for (long long c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
        unsigned long long idx = base, cv = (unsigned long long)c, cm = comp;
        while (cm) {
            const int g = __ffsll((long long)cm) - 1;
            cm &= cm - 1;
            idx |= (cv & 1ull) << g;
            cv >>= 1;
        }
        const typename V2<Real>::T v = s[idx];
        p += (double)v.x * v.x + (double)v.y * v.y;
    }
    p = warp_sum(p);
    __shared__ double sh[RED_THREADS / 32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = p;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < RED_THREADS / 32; k++) t += sh[k];
        partial[blockIdx.x] = t;
    }
}

__global__ void marginal_chunks_final(const double *partial, long long M, int nch, double *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double b = -1.0;
        long long bi = 0;
        for (long long x = 0; x < M; x++) {
            double p = 0.0;
            for (int k = 0; k < nch; k++) p += partial[x * nch + k];
            if (p > b) {  // lowest value on ties
                b = p;
                bi = x;
            }
        }
        out[0] = b;
        out[1] = (double)bi;
    }
}

// Queues the marginal argmax of `mask` over state s: its probability and
// value land in out[0], out[1].  Scratch: pbest / ibest of RED_BLOCKS entries.
static int queue_marginal(State *s, uint64_t mask, double *pbest, long long *ibest, double *out, cudaStream_t st) {
    const int n = s->qubits;
    if (n < 64 && (mask >> n)) return fail(HGM_ERR_INVALID, "mask beyond state bits");
    const int m = __builtin_popcountll(mask);
    const long long M = 1ll << m;
    if (M <= RED_BLOCKS) {
        const int nch = (int)(RED_BLOCKS / M);
        const unsigned g = (unsigned)(M * nch);
        if (s->precision == HGM_F64)
            marginal_chunk_kernel<double><<<g, RED_THREADS, 0, st>>>((const double2 *)s->d, n, mask, nch, pbest);
        else
            marginal_chunk_kernel<float><<<g, RED_THREADS, 0, st>>>((const float2 *)s->d, n, mask, nch, pbest);
        marginal_chunks_final<<<1, 32, 0, st>>>(pbest, M, nch, out);
    } else {
        unsigned g = (unsigned)((M + RED_THREADS - 1) / RED_THREADS);
        if (g > RED_BLOCKS) g = RED_BLOCKS;
        if (s->precision == HGM_F64)
            marginal_kernel<double><<<g, RED_THREADS, 0, st>>>((const double2 *)s->d, n, mask, m, pbest, ibest);
        else
            marginal_kernel<float><<<g, RED_THREADS, 0, st>>>((const float2 *)s->d, n, mask, m, pbest, ibest);
        marginal_final<<<1, 32, 0, st>>>(pbest, ibest, (int)g, out);
    }
    count_launch(2);
    return check("argmax launch");
}

// The whole marginal distribution over the bits of `mask` (DGM::measure(vector),
// src/core/dgm_core.cpp:150-162): out[x] = sum over the other bits of |a|^2,
// for every value x of the mask bits (bit j of x is the j-th lowest mask bit).
__global__ void marginal_chunks_sum(const double *partial, long long M, int nch, double *out) {
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < M; x += (long long)gridDim.x * blockDim.x) {
        double p = 0.0;
        for (int k = 0; k < nch; k++) p += partial[x * nch + k];
        out[x] = p;
    }
}

template <typename Real>
__global__ void __launch_bounds__(RED_THREADS) marginal_values_kernel(const typename V2<Real>::T *__restrict__ s, int n,
                                                                       unsigned long long mask, int m, double *out) {
    const unsigned long long comp = ~mask & ((n >= 64) ? ~0ull : ((1ull << n) - 1));
    const long long M = 1ll << m, C = 1ll << (n - m);
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < M; x += (long long)gridDim.x * blockDim.x) {
        unsigned long long base = 0, src = (unsigned long long)x, mm = mask;
        while (mm) {
            const int g = __ffsll((long long)mm) - 1;
            mm &= mm - 1;
            base |= (src & 1ull) << g;
            src >>= 1;
        }
        double p = 0.0;
        for (long long c = 0; c < C; c++) {
            unsigned long long idx = base, cs = (unsigned long long)c, cm = comp;
            while (cm) {
                const int g = __ffsll((long long)cm) - 1;
                cm &= cm - 1;
                idx |= (cs & 1ull) << g;
                cs >>= 1;
            }
            const typename V2<Real>::T v = s[idx];
            p += (double)v.x * v.x + (double)v.y * v.y;
        }
        out[x] = p;
    }
}

int marginal_probs(State *s, uint64_t mask, double *host_out, void *stream) {
    if (ensure_ctx()) return HGM_ERR_CUDA;
    cudaStream_t st = pick(stream);
    if (!st) return HGM_ERR_CUDA;
    const int n = s->qubits;
    if (n < 64 && (mask >> n)) return fail(HGM_ERR_INVALID, "mask beyond state bits");
    const int m = __builtin_popcountll(mask);
    if (m > 26) return fail(HGM_ERR_UNSUPPORTED, "marginal over %d bits (at most 26)", m);
    const long long M = 1ll << m;
    double *d_out = nullptr;
    cudaError_t e = cudaMallocAsync(&d_out, (size_t)M * sizeof(double), st);
    if (e != cudaSuccess) return fail(HGM_ERR_NOMEM, "marginal output: %s", cudaGetErrorString(e));
    if (M <= RED_BLOCKS) {
        const int nch = (int)(RED_BLOCKS / M);
        const unsigned g = (unsigned)(M * nch);
        if (s->precision == HGM_F64)
            marginal_chunk_kernel<double><<<g, RED_THREADS, 0, st>>>((const double2 *)s->d, n, mask, nch, g_ctx.partials);
        else
            marginal_chunk_kernel<float><<<g, RED_THREADS, 0, st>>>((const float2 *)s->d, n, mask, nch, g_ctx.partials);
        marginal_chunks_sum<<<(unsigned)((M + 255) / 256), 256, 0, st>>>(g_ctx.partials, M, nch, d_out);
    } else {
        unsigned g = (unsigned)((M + RED_THREADS - 1) / RED_THREADS);
        if (g > RED_BLOCKS) g = RED_BLOCKS;
        if (s->precision == HGM_F64)
            marginal_values_kernel<double><<<g, RED_THREADS, 0, st>>>((const double2 *)s->d, n, mask, m, d_out);
        else
            marginal_values_kernel<float><<<g, RED_THREADS, 0, st>>>((const float2 *)s->d, n, mask, m, d_out);
    }
    count_launch(2);
    int rc = check("marginal probabilities launch");
    if (!rc) {
        e = cudaMemcpyAsync(host_out, d_out, (size_t)M * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = fail(HGM_ERR_CUDA, "marginal probabilities: %s", cudaGetErrorString(e));
    }
    cudaFreeAsync(d_out, st);
    return rc;
}

int launch_argmax_async(State *s, uint64_t mask, double *pbest, long long *ibest, double *out, void *stream) {
    return queue_marginal(s, mask, pbest, ibest, out, (cudaStream_t)stream);
}

int marginal_argmax(State *s, uint64_t mask, int64_t *arg, double *prob, void *stream) {
    cudaStream_t st = pick(stream);
    if (!st) return HGM_ERR_CUDA;
    const int rc = queue_marginal(s, mask, g_ctx.partials, g_ctx.partial_idx, g_ctx.result, st);
    if (rc) return rc;
    cudaMemcpyAsync(g_ctx.host_result, g_ctx.result, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(HGM_ERR_CUDA, "marginal argmax: %s", cudaGetErrorString(e));
    if (prob) *prob = g_ctx.host_result[0];
    if (arg) *arg = (int64_t)g_ctx.host_result[1];
    return HGM_OK;
}


// ---------------------------------------------------------------------------
// Allocation-free FP64 norm (hgm_norm_noalloc)
// ---------------------------------------------------------------------------
// Some callers cannot allocate device memory: code embedded in a host
// framework that owns every device allocation (a plugin handed pre-allocated
// buffers), or code running while a CUDA graph is being captured elsewhere
// in the process, where a cudaMalloc would be illegal or would synchronise.
// Such a caller should queue it on a stream created non-blocking: the legacy
// default stream (stream NULL) synchronises with blocking streams, and a
// launch there while one of them captures invalidates that capture.
// This variant of the FP64 norm reduction keeps its per-block partial sums in
// a file-scope device array, so it allocates nothing: the caller passes the
// state and a device location for the result.
//
// Limits and sharing:
//   * the array holds NOALLOC_PARTIALS = 2*1184 doubles (18.5 KiB) on every
//     GPU that loads this library, for the life of the process;
//   * the reduction grid is capped at 1184 blocks (one partial each) for any
//     state size, so the array never limits the size; the qubit range
//     1..34 is the engine's own state range (hgm_state_create), and more
//     qubits are rejected with HGM_ERR_UNSUPPORTED;
//   * the result is exactly one double at d_out: the final step writes
//     d_out[0] and nothing after it;
//   * every call shares the array; each call writes every partial it reads
//     before reading it, so nothing needs clearing, but calls that overlap
//     on the GPU (different streams, or different host threads) race on it
//     and must be serialised by the caller;
//   * the array's device address is looked up once per device, on the first
//     call with that device current (cudaGetSymbolAddress); make that first
//     call before any stream capture.
constexpr int NOALLOC_PARTIALS = 2 * RED_BLOCKS;
static __device__ __align__(256) double g_noalloc_partials[NOALLOC_PARTIALS];

// Final step of the allocation-free norm: sums the block partials in the same
// fixed order as reduce_final and writes the one result double.
__global__ void noalloc_norm_final(const double *partials, int nblocks, double *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double t0 = 0.0;
        for (int k = 0; k < nblocks; k++) t0 += partials[2 * k];
        out[0] = t0;
    }
}

namespace {
std::mutex g_noalloc_mu;
double *g_noalloc_ptr[64] = {};
}  // namespace

static int noalloc_scratch(double **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(HGM_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return fail(HGM_ERR_UNSUPPORTED, "device %d beyond 64", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess) return fail(HGM_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        g_noalloc_ptr[dev] = reinterpret_cast<double *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return HGM_OK;
}

}  // namespace hgm

using namespace hgm;

extern "C" int hgm_norm_noalloc(const void *d_state, int qubits, int precision, double *d_out, void *stream) {
    if (!d_state || !d_out) return fail(HGM_ERR_INVALID, "null state or output pointer");
    if (precision != HGM_F64 && precision != HGM_F32) return fail(HGM_ERR_INVALID, "bad precision");
    if (qubits < 1 || qubits > 34)
        return fail(HGM_ERR_UNSUPPORTED, "qubits=%d outside 1..34, the engine's state range", qubits);
    double *partials = nullptr;
    int rc = noalloc_scratch(&partials);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;  // NULL: the legacy default stream
    const long long N = 1ll << qubits;
    const unsigned g = grid_for(N);
    if (precision == HGM_F64)
        reduce_kernel<double, double, RED_NORM><<<g, RED_THREADS, 0, st>>>((const double2 *)d_state, nullptr, N, 0,
                                                                            partials);
    else
        reduce_kernel<float, float, RED_NORM><<<g, RED_THREADS, 0, st>>>((const float2 *)d_state, nullptr, N, 0,
                                                                          partials);
    noalloc_norm_final<<<1, 32, 0, st>>>(partials, (int)g, d_out);
    count_launch(2);
    return check("hgm_norm_noalloc launch");
}

namespace hgm {
}  // namespace hgm

using namespace hgm;

extern "C" {

int64_t hgm_kernel_launches(void) { return g_launches.load(); }

int hgm_timer_start(void) {
    if (ensure_ctx()) return HGM_ERR_CUDA;
    cudaError_t e = cudaEventRecord(g_ctx.t0, g_ctx.stream);
    return e == cudaSuccess ? HGM_OK : fail(HGM_ERR_CUDA, "event record: %s", cudaGetErrorString(e));
}

int hgm_timer_stop(double *ms) {
    if (ensure_ctx()) return HGM_ERR_CUDA;
    cudaEventRecord(g_ctx.t1, g_ctx.stream);
    cudaError_t e = cudaEventSynchronize(g_ctx.t1);
    if (e != cudaSuccess) return fail(HGM_ERR_CUDA, "event sync: %s", cudaGetErrorString(e));
    float f = 0;
    cudaEventElapsedTime(&f, g_ctx.t0, g_ctx.t1);
    if (ms) *ms = f;
    return HGM_OK;
}

}  // extern "C"
