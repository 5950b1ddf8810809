// Test-only harness around the reference's own DGM engine.
//
// This file is oracle infrastructure: it is compiled by oracle/build_ref.sh
// together with the reference's unmodified (FP32) or type-widened (FP64)
// core sources into oracle/_ref/libref_*.so, and is only ever loaded by the
// test suite, the golden-fixture generator and bench.py's CPU-baseline leg.
// Nothing in the product links it.
//
// It exposes a flat C interface over the reference's DGM class
// (include/core/dgm.h:65-163) so Python can drive the reference exactly the
// way its own algorithm libraries do: register gates (Gates::addGate,
// src/core/gates.cpp:49-60), parse circuit strings (DGM::setFunction,
// src/core/dgm_parser.cpp:29-66), execute on a chosen backend
// (DGM::execute, src/core/dgm_core.cpp:243-267) and read the state back.
//
// REF_REAL is float for the unmodified reference and double for the widened
// copy; the reference's headers define `complex` as `__complex__`.
#include "core/dgm.h"
#include "core/gates.h"
#include <cstring>
#include <cstdint>
#include <random>
#include <vector>

#ifndef REF_REAL
#error "REF_REAL must be defined (float or double)"
#endif

typedef REF_REAL ref_real;
typedef ref_real __complex__ ref_cplx;

extern "C" {

int ref_amp_bytes(void) { return (int)sizeof(ref_cplx); }

void *ref_dgm_new(int qubits) {
    DGM *dgm = new DGM();
    dgm->qubits = qubits;
    // TuningDefaults (include/cli/cli_common.h:8-17)
    dgm->thread_count = 1;
    dgm->cpu_region_bits = 14;
    dgm->cpu_coalesced_bits = 11;
    dgm->gpu_count = 1;
    dgm->gpu_region_bits = 8;
    dgm->gpu_coalesced_bits = 4;
    dgm->block_size = 64;
    dgm->repeat_count = 2;
    dgm->allocateMemory();
    return dgm;
}

void ref_dgm_free(void *h) { delete (DGM *)h; }

void ref_dgm_set_tuning(void *h, int exec_type, int thread_count, int cpu_region_bits,
                        int cpu_coalesced_bits, int gpu_count, int gpu_region_bits,
                        int gpu_coalesced_bits, int block_size, int repeat_count) {
    DGM *dgm = (DGM *)h;
    dgm->exec_type = exec_type;
    dgm->thread_count = thread_count;
    dgm->cpu_region_bits = cpu_region_bits;
    dgm->cpu_coalesced_bits = cpu_coalesced_bits;
    dgm->gpu_count = gpu_count;
    dgm->gpu_region_bits = gpu_region_bits;
    dgm->gpu_coalesced_bits = gpu_coalesced_bits;
    dgm->block_size = block_size;
    dgm->repeat_count = repeat_count;
}

// m: 8 doubles, row-major [m00, m01, m10, m11] as (re, im) pairs.
int ref_dgm_add_gate(void *h, const char *name, const double *m) {
    DGM *dgm = (DGM *)h;
    ref_cplx a[4];
    for (int i = 0; i < 4; i++) {
        __real__ a[i] = (ref_real)m[2 * i];
        __imag__ a[i] = (ref_real)m[2 * i + 1];
    }
    return dgm->gates.addGate(name, a[0], a[1], a[2], a[3]) ? 1 : 0;
}

void ref_dgm_set_memory_value(void *h, long pos) {
    DGM *dgm = (DGM *)h;
    memset(dgm->state, 0, sizeof(ref_cplx) * (1L << dgm->qubits));
    dgm->setMemoryValue((int)pos);
}

void ref_dgm_set_state(void *h, const double *amps) {
    DGM *dgm = (DGM *)h;
    long size = 1L << dgm->qubits;
    for (long i = 0; i < size; i++) {
        __real__ dgm->state[i] = (ref_real)amps[2 * i];
        __imag__ dgm->state[i] = (ref_real)amps[2 * i + 1];
    }
}

void ref_dgm_get_state(void *h, double *amps) {
    DGM *dgm = (DGM *)h;
    long size = 1L << dgm->qubits;
    for (long i = 0; i < size; i++) {
        amps[2 * i] = (double)__real__ dgm->state[i];
        amps[2 * i + 1] = (double)__imag__ dgm->state[i];
    }
}

// steps: ';'-separated circuit steps, exactly as DGM::setFunction(string).
void ref_dgm_set_function(void *h, const char *steps, int iterations, int reset) {
    DGM *dgm = (DGM *)h;
    long keep = dgm->qubits;
    dgm->setFunction(std::string(steps), iterations, reset != 0);
    dgm->qubits = keep;
}

long ref_dgm_num_pts(void *h) {
    DGM *dgm = (DGM *)h;
    if (!dgm->pts) return 0;
    long n = 0;
    while (dgm->pts[n] != NULL) n++;
    return n;
}

// Dumps the compiled PT list: per PT, target_bit, control_mask, control_value
// and the 2x2 matrix widened to double.
void ref_dgm_dump_pts(void *h, int32_t *target, int64_t *cmask, int64_t *cval, double *mat) {
    DGM *dgm = (DGM *)h;
    for (long i = 0; dgm->pts[i] != NULL; i++) {
        PT *pt = dgm->pts[i];
        target[i] = pt->target_bit;
        cmask[i] = pt->control_mask;
        cval[i] = pt->control_value;
        for (int k = 0; k < 4; k++) {
            mat[8 * i + 2 * k] = (double)__real__ pt->matrix[k];
            mat[8 * i + 2 * k + 1] = (double)__imag__ pt->matrix[k];
        }
    }
}

// Runs DGM::execute on the backend chosen by ref_dgm_set_tuning.
void ref_dgm_execute(void *h, int iterations) {
    DGM *dgm = (DGM *)h;
    dgm->execute(iterations);
}

void ref_seed_rng(unsigned long seed) { seed_rng(seed); }

int ref_dgm_measure(void *h, int qubit) { return ((DGM *)h)->measure(qubit); }

// The uniform sample DGM::measure(int) draws first after seed_rng(seed)
// (src/core/dgm_core.cpp:97-101: a uniform_real_distribution<double>(0, 1) on
// g_rng); g_rng is re-seeded with `seed` afterwards, so the next measure draws
// the same value.
double ref_uniform_sample(unsigned long seed) {
    seed_rng(seed);
    std::uniform_real_distribution<double> dist(0.0, 1.0);
    const double v = dist(g_rng);
    seed_rng(seed);
    return v;
}

// DGM::colapse(qubit, value) (src/core/dgm_core.cpp:129-146).
void ref_dgm_colapse(void *h, int qubit, int value) { ((DGM *)h)->colapse(qubit, value); }

// DGM::measure(vector<int>) (src/core/dgm_core.cpp:150-162): its map's keys
// (index & mask) and probabilities, in key order; returns the map's size.
long ref_dgm_measure_many(void *h, const int *qubits, int nq, long *keys, double *probs, long cap) {
    std::vector<int> pos(qubits, qubits + nq);
    auto m = ((DGM *)h)->measure(pos);
    long k = 0;
    for (auto &kv : m) {
        if (k < cap) {
            keys[k] = kv.first;
            probs[k] = (double)kv.second;
        }
        k++;
    }
    return k;
}

}  // extern "C"
