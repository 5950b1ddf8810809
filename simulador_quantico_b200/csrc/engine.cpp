// C-ABI of the engine: runtime, plans, device states, execution and
// device-resident measurement (include/hgm_b200.h).
#include <cuda_runtime.h>

#include <cstdlib>

#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>

#include "hgm_dropin_layout.h"
#include "hgm_internal.h"

using namespace hgm;

namespace {

int cuda_fail(cudaError_t e, const char *what) {
    return fail(e == cudaErrorMemoryAllocation ? HGM_ERR_NOMEM : HGM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

template <typename Real>
void ops_from_ref_pts(void *const *pts, std::vector<Op> &out) {
    for (long i = 0; pts[i] != nullptr; i++) {
        const RefPTLayout *pt = reinterpret_cast<const RefPTLayout *>(pts[i]);
        const Real *m = reinterpret_cast<const Real *>(pt->matrix);
        Op op;
        op.target = pt->target_bit;
        op.cmask = (uint64_t)pt->control_mask;
        op.cval = (uint64_t)pt->control_value;
        for (int k = 0; k < 4; k++) op.m[k] = cplx((double)m[2 * k], (double)m[2 * k + 1]);
        out.push_back(op);
    }
}

}  // namespace

namespace {
std::mutex g_lease_mu;

void free_plan_now(Plan *pl) {
    // launches are asynchronous: the plan's device records may still be in use
    if (pl->d_ops || pl->d_phases) cudaDeviceSynchronize();
    delete pl;
}
}  // namespace

namespace hgm {
void plan_lease(const Plan *plan) {
    std::lock_guard<std::mutex> lk(g_lease_mu);
    const_cast<Plan *>(plan)->leases++;
}
void plan_unlease(const Plan *plan) {
    Plan *pl = const_cast<Plan *>(plan);
    bool now = false;
    {
        std::lock_guard<std::mutex> lk(g_lease_mu);
        now = --pl->leases == 0 && pl->free_pending;
    }
    if (now) free_plan_now(pl);
}
}  // namespace hgm

extern "C" {

int hgm_init(int device) {
    // The server runs up to 16 streams; with the driver's default of 8
    // hardware queues, two streams share a queue and a long pass on one holds
    // back the other's kernels (served throughput swung between 183 and 264
    // circuits/s with 8, held at 266-268 with 32).  Takes effect only if no
    // CUDA context exists yet in this process; a value the user set stays.
    setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    e = cudaFree(0);
    if (e != cudaSuccess) return cuda_fail(e, "context init");
    return default_stream() ? HGM_OK : HGM_ERR_CUDA;
}

int hgm_synchronize(void) {
    cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? HGM_OK : cuda_fail(e, "cudaDeviceSynchronize");
}

int hgm_pinned_alloc(int64_t bytes, void **out) {
    if (!out || bytes <= 0) return fail(HGM_ERR_INVALID, "bad pinned allocation request");
    cudaError_t e = cudaMallocHost(out, (size_t)bytes);
    return e == cudaSuccess ? HGM_OK : cuda_fail(e, "cudaMallocHost");
}

void hgm_pinned_free(void *p) {
    if (p) cudaFreeHost(p);
}

int hgm_mem_info(int64_t *free_bytes, int64_t *total_bytes) {
    size_t f = 0, t = 0;
    cudaError_t e = cudaMemGetInfo(&f, &t);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemGetInfo");
    if (free_bytes) *free_bytes = (int64_t)f;
    if (total_bytes) *total_bytes = (int64_t)t;
    return HGM_OK;
}

void hgm_plan_default_opts(hgm_plan_opts *o, int precision) {
    o->precision = precision;
    o->warp_bits = -1;
    o->low_bits = -1;
    o->fuse = 1;
    o->window = 0;
    o->renorm_every = precision == HGM_F32 ? 64 : 0;
    o->chained = 1;
    // both precisions (FP64 saves 2 of 8 instructions per amplitude: 26- to
    // 30-qubit FP64 layered circuits 3-4% faster)
    o->split_layers = 1;
    o->reg_bits = -1;
}

static int finish_plan(const std::vector<Op> &ops, int qubits, const hgm_plan_opts *opts, hgm_plan **out) {
    if (!out) return fail(HGM_ERR_INVALID, "null output");
    hgm_plan_opts o;
    if (opts) o = *opts;
    else hgm_plan_default_opts(&o, HGM_F64);
    if (o.precision != HGM_F64 && o.precision != HGM_F32) return fail(HGM_ERR_INVALID, "bad precision");
    std::unique_ptr<Plan> p(new Plan());
    int rc = build_plan(ops, qubits, o, p.get());
    if (rc) return rc;
    *out = reinterpret_cast<hgm_plan *>(p.release());
    return HGM_OK;
}

int hgm_plan_create(const hgm_circuit *c, int qubits, const hgm_plan_opts *opts, hgm_plan **out) {
    if (!c) return fail(HGM_ERR_INVALID, "null circuit");
    return finish_plan(reinterpret_cast<const Circuit *>(c)->ops, qubits, opts, out);
}

int hgm_plan_create_from_ref_pts(void *const *pts, int pt_precision, int qubits, const hgm_plan_opts *opts,
                                 hgm_plan **out) {
    if (!pts) return fail(HGM_ERR_INVALID, "null PT list");
    std::vector<Op> ops;
    if (pt_precision == HGM_F64) ops_from_ref_pts<double>(pts, ops);
    else ops_from_ref_pts<float>(pts, ops);
    return finish_plan(ops, qubits, opts, out);
}


void hgm_plan_free(hgm_plan *p) {
    Plan *pl = reinterpret_cast<Plan *>(p);
    if (!pl) return;
    {
        // a plan that queued server requests still use is freed by the last of them
        std::lock_guard<std::mutex> lk(g_lease_mu);
        if (pl->leases > 0) {
            pl->free_pending = true;
            return;
        }
    }
    free_plan_now(pl);
}

int hgm_plan_upload(hgm_plan *p) {
    if (!p) return fail(HGM_ERR_INVALID, "null plan");
    return upload_plan(reinterpret_cast<Plan *>(p));
}

int hgm_plan_stats(const hgm_plan *p, int64_t *n_ops, int64_t *n_passes, int64_t *n_phases, int64_t *n_transposes) {
    if (!p) return fail(HGM_ERR_INVALID, "null plan");
    const Plan *pl = reinterpret_cast<const Plan *>(p);
    if (n_ops) *n_ops = pl->n_ops;
    if (n_passes) *n_passes = pl->small ? (pl->n_small_ops ? 1 : 0) : (int64_t)pl->passes.size();
    if (n_phases) *n_phases = (int64_t)pl->phases.size();
    if (n_transposes) *n_transposes = pl->n_transposes;
    return HGM_OK;
}

int hgm_plan_layouts(const hgm_plan *p, const int8_t **pos, int64_t *n_layouts) {
    const Plan *pl = reinterpret_cast<const Plan *>(p);
    if (!pl) return fail(HGM_ERR_INVALID, "null plan");
    if (pos) *pos = pl->layouts.empty() ? nullptr : pl->layouts[0].pos;
    if (n_layouts) *n_layouts = (int64_t)pl->layouts.size();
    return HGM_OK;
}

int hgm_plan_export(const hgm_plan *p, const void **passes, int64_t *n_passes, const void **phases,
                    int64_t *n_phases, const void **ops, int64_t *ops_bytes, int *warp_bits, int *small) {
    if (!p) return fail(HGM_ERR_INVALID, "null plan");
    const Plan *pl = reinterpret_cast<const Plan *>(p);
    if (passes) *passes = pl->passes.data();
    if (n_passes) *n_passes = (int64_t)pl->passes.size();
    if (phases) *phases = pl->phases.data();
    if (n_phases) *n_phases = (int64_t)pl->phases.size();
    if (ops) *ops = pl->ops_bytes.data();
    if (ops_bytes) *ops_bytes = (int64_t)pl->ops_bytes.size();
    if (warp_bits) *warp_bits = pl->warp_bits;
    if (small) *small = pl->small ? 1 : 0;
    return HGM_OK;
}

int hgm_state_create(int qubits, int precision, hgm_state **out) {
    if (!out) return fail(HGM_ERR_INVALID, "null output");
    if (qubits < 1 || qubits > 34) return fail(HGM_ERR_UNSUPPORTED, "qubits=%d outside 1..34", qubits);
    if (precision != HGM_F64 && precision != HGM_F32) return fail(HGM_ERR_INVALID, "bad precision");
    if (!default_stream()) return HGM_ERR_CUDA;
    std::unique_ptr<State> s(new State());
    s->qubits = qubits;
    s->precision = precision;
    cudaError_t e = cudaMalloc(&s->d, (size_t)s->bytes());
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(e, "state allocation");
    }
    *out = reinterpret_cast<hgm_state *>(s.release());
    return HGM_OK;
}

void hgm_state_free(hgm_state *s) {
    State *st = reinterpret_cast<State *>(s);
    if (!st || !st->owned) return;  // views are released by their owner
    if (st->d) {
        cudaDeviceSynchronize();  // work queued on the state may still be running
        cudaFree(st->d);
    }
    delete st;
}

int hgm_state_qubits(const hgm_state *s) { return s ? reinterpret_cast<const State *>(s)->qubits : 0; }
int hgm_state_precision(const hgm_state *s) { return s ? reinterpret_cast<const State *>(s)->precision : -1; }
void *hgm_state_device_ptr(hgm_state *s) { return s ? reinterpret_cast<State *>(s)->d : nullptr; }

int hgm_state_set_basis(hgm_state *s, int64_t index) {
    if (!s) return fail(HGM_ERR_INVALID, "null state");
    return launch_set_basis(reinterpret_cast<State *>(s), index, nullptr);
}

int hgm_state_upload(hgm_state *s, const void *host, int64_t bytes) {
    State *st = reinterpret_cast<State *>(s);
    if (!st || !host) return fail(HGM_ERR_INVALID, "null argument");
    if (bytes != st->bytes()) return fail(HGM_ERR_INVALID, "upload of %lld bytes into a %lld-byte state",
                                          (long long)bytes, (long long)st->bytes());
    return copy_state(st->d, host, (size_t)bytes, true, default_stream());
}

int hgm_state_download(const hgm_state *s, void *host, int64_t bytes) {
    const State *st = reinterpret_cast<const State *>(s);
    if (!st || !host) return fail(HGM_ERR_INVALID, "null argument");
    if (bytes != st->bytes()) return fail(HGM_ERR_INVALID, "download of %lld bytes from a %lld-byte state",
                                          (long long)bytes, (long long)st->bytes());
    return copy_state(host, st->d, (size_t)bytes, false, default_stream());
}

int hgm_execute(hgm_state *s, const hgm_plan *p, int iterations, void *stream) {
    if (!s || !p) return fail(HGM_ERR_INVALID, "null argument");
    if (iterations < 0) return fail(HGM_ERR_INVALID, "negative iterations");
    Plan *pl = const_cast<Plan *>(reinterpret_cast<const Plan *>(p));
    int rc = upload_plan(pl);
    if (rc) return rc;
    if (iterations == 0) return HGM_OK;
    // a state that fits in L2 runs every pass in one chained launch
    if (plan_launches(pl, iterations) > 1 && chain_eligible(pl, iterations))
        return launch_plan_chain(reinterpret_cast<State *>(s), pl, iterations, stream);
    return launch_plan(reinterpret_cast<State *>(s), pl, iterations, stream);
}

int hgm_plan_status(const hgm_plan *p) {
    if (!p) return fail(HGM_ERR_INVALID, "null plan");
    const Plan *pl = reinterpret_cast<const Plan *>(p);
    const void *w = chain_error_word(pl);
    if (!w) return HGM_OK;
    uint64_t err = 0;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&err, w, sizeof err, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "plan status");
    return err ? fail(HGM_ERR_TIMEOUT, "a chained pass gave up waiting for the passes before it") : HGM_OK;
}

int hgm_norm(hgm_state *s, double *out) {
    if (!s) return fail(HGM_ERR_INVALID, "null state");
    return reduce_norm(reinterpret_cast<State *>(s), out, nullptr);
}

int hgm_prob_one(hgm_state *s, int bit, double *out) {
    if (!s) return fail(HGM_ERR_INVALID, "null state");
    return reduce_prob_one(reinterpret_cast<State *>(s), bit, out, nullptr);
}

int hgm_measure_qubit(hgm_state *s, int qubit, double sample, int *outcome, double *prob) {
    State *st = reinterpret_cast<State *>(s);
    if (!st) return fail(HGM_ERR_INVALID, "null state");
    if (qubit < 0 || qubit >= st->qubits) return fail(HGM_ERR_INVALID, "qubit %d outside state", qubit);
    const int bit = st->qubits - 1 - qubit;
    double total = 0, one = 0;
    int rc = reduce_norm(st, &total, nullptr);
    if (!rc) rc = reduce_prob_one(st, bit, &one, nullptr);
    if (rc) return rc;
    const double zero = total - one;
    // DGM::measure: outcome 0 iff P(0) > sample (dgm_core.cpp:97-113)
    const int value = (zero > sample) ? 0 : 1;
    const double p = value ? one : zero;
    if (!(p > 0)) return fail(HGM_ERR_INVALID, "measured outcome has zero probability");
    // the measured branch, rescaled, moves to the qubit's |0> half
    // (dgm_core.cpp:117-122)
    rc = measure_update(st, bit, value, 1.0 / std::sqrt(p), nullptr);
    if (rc) return rc;
    if (outcome) *outcome = value;
    if (prob) *prob = p;
    return HGM_OK;
}

int hgm_collapse_qubit(hgm_state *s, int qubit, int value, double *prob) {
    State *st = reinterpret_cast<State *>(s);
    if (!st) return fail(HGM_ERR_INVALID, "null state");
    if (qubit < 0 || qubit >= st->qubits) return fail(HGM_ERR_INVALID, "qubit %d outside state", qubit);
    if (value != 0 && value != 1) return fail(HGM_ERR_INVALID, "value %d is not 0 or 1", value);
    const int bit = st->qubits - 1 - qubit;
    double total = 0, one = 0;
    int rc = reduce_norm(st, &total, nullptr);
    if (!rc) rc = reduce_prob_one(st, bit, &one, nullptr);
    if (rc) return rc;
    const double p = value ? one : total - one;
    if (!(p > 0)) return fail(HGM_ERR_INVALID, "collapse onto a value of zero probability");
    // DGM::colapse (dgm_core.cpp:129-146): keep the amplitudes whose qubit has
    // `value`, divide them by sqrt of their probability, clear the rest
    rc = collapse(st, bit, value, 1.0 / std::sqrt(p), nullptr);
    if (rc) return rc;
    if (prob) *prob = p;
    return HGM_OK;
}

int hgm_marginal_probs(hgm_state *s, uint64_t mask, double *out, int64_t count) {
    State *st = reinterpret_cast<State *>(s);
    if (!st || !out) return fail(HGM_ERR_INVALID, "null argument");
    const int m = __builtin_popcountll(mask);
    if (m > 62 || count != (int64_t(1) << m))
        return fail(HGM_ERR_INVALID, "output holds %lld values, the mask needs 2^%d", (long long)count, m);
    return marginal_probs(st, mask, out, nullptr);
}

int hgm_marginal_argmax(hgm_state *s, uint64_t mask, int64_t *arg, double *prob) {
    if (!s) return fail(HGM_ERR_INVALID, "null state");
    return marginal_argmax(reinterpret_cast<State *>(s), mask, arg, prob, nullptr);
}

int hgm_inner(hgm_state *a, hgm_state *b, double *re, double *im) {
    if (!a || !b) return fail(HGM_ERR_INVALID, "null state");
    return inner(reinterpret_cast<State *>(a), reinterpret_cast<State *>(b), re, im, nullptr);
}

int hgm_max_abs_diff(hgm_state *a, hgm_state *b, double *out) {
    if (!a || !b) return fail(HGM_ERR_INVALID, "null state");
    return max_abs_diff(reinterpret_cast<State *>(a), reinterpret_cast<State *>(b), out, nullptr);
}

int hgm_scale(hgm_state *s, double f) {
    if (!s) return fail(HGM_ERR_INVALID, "null state");
    return scale_state(reinterpret_cast<State *>(s), f, nullptr);
}

}  // extern "C"
