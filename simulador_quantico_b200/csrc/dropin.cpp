// The reference's GPU-backend C-ABI on top of the engine (include/hgm_dropin.h).
//
// Compiled twice: without HGM_DROPIN_F64 into libhgm_dropin_f32.so (for the
// unmodified, FP32 reference) and with it into libhgm_dropin_f64.so (for the
// FP64-widened reference).  Replaces the reference's src/core/kernel.cu at
// link time (makefile:51-61).
//
// Call semantics kept from src/core/kernel.cu:131-316: the host state is
// copied in, the PT list is applied `iterations` times, the state is copied
// back in place and the same pointer is returned; any failure prints a
// message and exits with status 1 (kernel.cu:439-447).  Unlike the
// reference, the device buffer is kept between calls of the same size and
// precision (one cudaMalloc per process instead of one per call), and the
// plans of the last few PT lists are kept: a call whose list has the same
// targets, controls and matrices as a cached one (compared in full, not by
// hash alone) runs that plan instead of planning the list again.  With
// HYBRID_DEBUG set (the reference's switch, kernel.cu:304-313) each call
// prints its elapsed time split into planning, copies and execution.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <map>
#include <mutex>
#include <vector>

#include "hgm_b200.h"
#include "hgm_dropin.h"

#ifdef HGM_DROPIN_F64
static const int kPrecision = HGM_F64;
#else
static const int kPrecision = HGM_F32;
#endif

namespace {

std::mutex g_mu;

// Device states kept between calls, by qubit count.  Callers that run many
// circuits of a few sizes (the batched comparison) would otherwise pay a
// device allocation and free per call, more than a small circuit's run.
// At most kKeepBytes are kept; a state that does not fit replaces the rest.
constexpr int64_t kKeepBytes = int64_t(4) << 30;
std::map<int, hgm_state *> g_states;
int64_t g_kept = 0;

hgm_state *state_for(int qubits) {
    auto it = g_states.find(qubits);
    if (it != g_states.end()) return it->second;
    const int64_t bytes = (int64_t(1) << qubits) * (int64_t)sizeof(hgm_dropin_amp);
    if (g_kept + bytes > kKeepBytes) {
        for (auto &kv : g_states) hgm_state_free(kv.second);
        g_states.clear();
        g_kept = 0;
    }
    hgm_state *st = nullptr;
    if (hgm_state_create(qubits, kPrecision, &st)) return nullptr;
    g_states[qubits] = st;
    g_kept += bytes;
    return st;
}

// Plans of recent PT lists, keyed by the list's content: per PT its target
// bit, control mask and value and its four matrix entries, as bytes.
constexpr size_t kPlanCache = 8;
struct CachedPlan {
    int qubits = 0;
    uint64_t hash = 0;
    std::vector<unsigned char> key;
    hgm_plan *plan = nullptr;
    uint64_t last_use = 0;
};
std::vector<CachedPlan> g_plans;
uint64_t g_use = 0;

void pt_key(hgm_ref_pt **pts, std::vector<unsigned char> &key, uint64_t &hash) {
    key.clear();
    for (long i = 0; pts[i] != nullptr; i++) {
        const hgm_ref_pt *pt = pts[i];
        const size_t at = key.size();
        key.resize(at + sizeof(int) + 2 * sizeof(long) + 4 * sizeof(hgm_dropin_amp));
        unsigned char *d = key.data() + at;
        memcpy(d, &pt->target_bit, sizeof(int));
        memcpy(d + sizeof(int), &pt->control_mask, sizeof(long));
        memcpy(d + sizeof(int) + sizeof(long), &pt->control_value, sizeof(long));
        memcpy(d + sizeof(int) + 2 * sizeof(long), pt->matrix, 4 * sizeof(hgm_dropin_amp));
    }
    uint64_t h = 1469598103934665603ull;  // FNV-1a
    for (unsigned char c : key) {
        h ^= c;
        h *= 1099511628211ull;
    }
    hash = h;
}

hgm_plan *plan_for(hgm_ref_pt **pts, int qubits);

[[noreturn]] void die(const char *what) {
    printf("hgm_b200: %s: %s\n", what, hgm_last_error());
    fflush(stdout);
    exit(1);
}

hgm_plan *plan_for(hgm_ref_pt **pts, int qubits) {
    static std::vector<unsigned char> key;
    uint64_t hash = 0;
    pt_key(pts, key, hash);
    for (CachedPlan &c : g_plans)
        if (c.qubits == qubits && c.hash == hash && c.key == key) {
            c.last_use = ++g_use;
            return c.plan;
        }
    hgm_plan_opts opts;
    hgm_plan_default_opts(&opts, kPrecision);
    hgm_plan *plan = nullptr;
    if (hgm_plan_create_from_ref_pts(reinterpret_cast<void *const *>(pts), kPrecision, qubits, &opts, &plan))
        die("planning");
    if (g_plans.size() >= kPlanCache) {
        auto old = std::min_element(g_plans.begin(), g_plans.end(),
                                    [](const CachedPlan &a, const CachedPlan &b) { return a.last_use < b.last_use; });
        hgm_plan_free(old->plan);  // waits for the device before freeing
        g_plans.erase(old);
    }
    CachedPlan c;
    c.qubits = qubits;
    c.hash = hash;
    c.key = key;
    c.plan = plan;
    c.last_use = ++g_use;
    g_plans.push_back(std::move(c));
    return plan;
}

}  // namespace

extern "C" {

bool setDevice(int device_id) { return hgm_init(device_id) != HGM_OK; }

hgm_dropin_amp *GpuExecutionWrapper(hgm_dropin_amp *read_memory, hgm_ref_pt **pts, int qubits, int coalesced_bits,
                                    int gpu_region_bits, int gpu_count, int block_size, int repeat_count,
                                    int iterations) {
    static const bool debug = getenv("HYBRID_DEBUG") != nullptr;
    auto t_start = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lk(g_mu);

    // DGM::validateTuning's three GPU rules (src/core/dgm_core.cpp:199-240),
    // kept at this edge for callers that bypass DGM::execute: the exit status
    // and the message's first words are the reference's.
    if (2L * block_size * repeat_count != (1L << gpu_region_bits)) {
        printf("Erro de tuning: 2*block_size*repeat_count (%ld) precisa ser igual a 2^gpu_region_bits (%ld)\n",
               2L * block_size * repeat_count, 1L << gpu_region_bits);
        exit(1);
    }
    if (gpu_region_bits < coalesced_bits) {
        printf("Erro de tuning: gpu_region_bits (%d) precisa ser >= gpu_coalesced_bits (%d)\n", gpu_region_bits,
               coalesced_bits);
        exit(1);
    }
    if (gpu_count > 4) {
        printf("Erro de tuning: gpu_count (%d) precisa ser <= 4\n", gpu_count);
        exit(1);
    }
    if (gpu_count > 1) {
        static bool told = false;
        if (!told) fprintf(stderr, "hgm_b200: gpu_count=%d requested; running on one GPU\n", gpu_count);
        told = true;
    }
    if (read_memory == nullptr) {
        printf("hgm_b200: device-resident (hybrid) states are not provided\n");
        exit(1);
    }
    if (pts == nullptr) die("null PT list");

    auto ms_since = [](std::chrono::steady_clock::time_point t0) {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };
    auto t_phase = std::chrono::steady_clock::now();
    hgm_plan *plan = plan_for(pts, qubits);
    const double plan_ms = ms_since(t_phase);
    hgm_state *state = state_for(qubits);
    if (!state) die("state allocation");
    const int64_t bytes = (int64_t(1) << qubits) * (int64_t)sizeof(hgm_dropin_amp);
    t_phase = std::chrono::steady_clock::now();
    if (hgm_state_upload(state, read_memory, bytes)) die("copy to device");
    const double h2d_ms = ms_since(t_phase);
    t_phase = std::chrono::steady_clock::now();
    if (hgm_execute(state, plan, iterations, nullptr)) die("execution");
    if (debug && hgm_synchronize()) die("execution");
    const double exec_ms = ms_since(t_phase);
    t_phase = std::chrono::steady_clock::now();
    if (hgm_state_download(state, read_memory, bytes)) die("copy to host");
    const double d2h_ms = ms_since(t_phase);
    if (hgm_plan_status(plan)) die("execution");  // a chained run that gave up a bounded wait

    if (debug) {
        int64_t n_ops = 0, n_passes = 0;
        hgm_plan_stats(plan, &n_ops, &n_passes, nullptr, nullptr);
        fprintf(stderr,
                "[GPUEXEC]   qubits=%d elapsed_ms=%.3f plan_ms=%.3f h2d_ms=%.3f exec_ms=%.3f d2h_ms=%.3f ops=%lld "
                "passes=%lld\n",
                qubits, ms_since(t_start), plan_ms, h2d_ms, exec_ms, d2h_ms, (long long)n_ops, (long long)n_passes);
    }
    return read_memory;
}

bool ProjectState(hgm_dropin_amp *, int, int, long, long, int) {
    fprintf(stderr, "hgm_b200: the hybrid CPU+GPU mode (ProjectState) is not provided.\n");
    return false;
}

bool GetState(hgm_dropin_amp *, int, int, long, long, int) {
    fprintf(stderr, "hgm_b200: the hybrid CPU+GPU mode (GetState) is not provided.\n");
    return false;
}

}  // extern "C"
