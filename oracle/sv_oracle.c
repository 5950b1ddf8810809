/*
 * sv_oracle.c -- CPU restatement of the HybriD-GM state-vector engine.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the CUDA path is
 * checked against; only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg load it.  The product never links or calls it.
 *
 * It restates, in plain C99, the two CPU backends of the reference
 * (MMullerdR/simulador_quantico):
 *
 *   oracle_serial_*   DGM::CpuExecution1 and its three kernels
 *                     (src/core/dgm_cpu_exec.cpp:11-126): one PT at a time
 *                     over the whole state, dispatching on PT::matrixType
 *                     (src/core/common.cpp:33-38).
 *   oracle_regions_*  PCpuExecution1 / compute_region / PCpuExecution1_0
 *                     (src/core/dgm_par_exec.cpp:11-253): the t_PAR_CPU
 *                     region planner and the per-region loops, OpenMP
 *                     parallel over region ids.
 *
 * plus FP64 reductions used by the checks (norm, per-qubit probability,
 * inner product).  Each amplitude is stored interleaved (re, im), index bit b
 * belongs to circuit qubit n-1-b (docs/01-arquitetura-geral.md), and an op is
 * applied iff (index & control_mask) == control_value, with the row-major
 * matrix [m00, m01, m10, m11] (src/core/kernel.cu:109-111).
 *
 * Compiled twice (REAL = double, and REAL = float under -DORACLE_F32) by
 * oracle/Makefile; the
 * suffix _f64 / _f32 names the amplitude type.  Built with the reference's
 * own engine flags (-O3 -fcx-limited-range, no FMA contraction) so the FP64
 * serial path reproduces the widened reference bit for bit.
 */
#include <complex.h>
#include <stdint.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORACLE_F32
#define REAL float
#define SFX(name) name##_f32
#else
#define REAL double
#define SFX(name) name##_f64
#endif

typedef REAL complex cplx;

/* One compiled 1-qubit gate (the fields of struct PT that the engines read,
 * include/core/common.h:57-90). */
typedef struct {
    int32_t target;       /* PT::target_bit */
    int32_t pad;
    int64_t cmask;        /* PT::control_mask */
    int64_t cval;         /* PT::control_value */
    double m[8];          /* row-major 2x2, (re, im) pairs */
} oracle_op;

enum { DENSE = 0, DIAG_PRI = 1, DIAG_SEC = 2 };

static void load_matrix(const oracle_op *op, cplx m[4]) {
    for (int k = 0; k < 4; k++) m[k] = (REAL)op->m[2 * k] + (REAL)op->m[2 * k + 1] * I;
}

/* PT::matrixType, src/core/common.cpp:33-38 (exact zero tests). */
static int matrix_type(const cplx m[4]) {
    if ((m[1] == 0.0) && (m[2] == 0.0)) return DIAG_PRI;
    else if ((m[0] == 0.0) && (m[3] == 0.0)) return DIAG_SEC;
    return DENSE;
}

/* ------------------------------------------------------------------ */
/* Serial engine: DGM::CpuExecution1 (dgm_cpu_exec.cpp:11-35).          */
/* ------------------------------------------------------------------ */

/* CpuExecution1_1, dgm_cpu_exec.cpp:39-70 */
static void serial_dense(cplx *state, const oracle_op *op, const cplx m[4], long mem_size) {
    long tmask = 1L << op->target;
    cplx tmp;
    if (!op->cmask) {
        long half = mem_size / 2;
        for (long pos = 0; pos < half; pos++) {
            long p0 = (pos * 2) - (pos & (tmask - 1));
            long p1 = p0 | tmask;
            tmp = m[0] * state[p0] + m[1] * state[p1];
            state[p1] = m[2] * state[p0] + m[3] * state[p1];
            state[p0] = tmp;
        }
    } else {
        long mask = ~(op->cmask | tmask);
        long inc = (~mask) + 1;
        for (long pos = 0; pos < mem_size; pos = (pos + inc) & mask) {
            long p0 = pos | op->cval;
            long p1 = p0 | tmask;
            tmp = m[0] * state[p0] + m[1] * state[p1];
            state[p1] = m[2] * state[p0] + m[3] * state[p1];
            state[p0] = tmp;
        }
    }
}

/* CpuExecution1_2, dgm_cpu_exec.cpp:75-91 */
static void serial_diag(cplx *state, const oracle_op *op, const cplx m[4], long mem_size) {
    long t = op->target;
    if (!op->cmask) {
        for (long pos = 0; pos < mem_size; pos++) state[pos] = m[((pos >> t) & 1) * 3] * state[pos];
    } else {
        long mask = ~(op->cmask);
        long inc = (~mask) + 1;
        for (long pos = 0; pos < mem_size; pos = (pos + inc) & mask) {
            long p0 = pos | op->cval;
            state[p0] = m[((p0 >> t) & 1) * 3] * state[p0];
        }
    }
}

/* CpuExecution1_3, dgm_cpu_exec.cpp:95-126 */
static void serial_antidiag(cplx *state, const oracle_op *op, const cplx m[4], long mem_size) {
    long tmask = 1L << op->target;
    cplx tmp;
    if (!op->cmask) {
        long half = mem_size / 2;
        for (long pos = 0; pos < half; pos++) {
            long p0 = (pos * 2) - (pos & (tmask - 1));
            long p1 = p0 | tmask;
            tmp = m[1] * state[p1];
            state[p1] = m[2] * state[p0];
            state[p0] = tmp;
        }
    } else {
        long mask = ~(op->cmask | tmask);
        long inc = (~mask) + 1;
        for (long pos = 0; pos < mem_size; pos = (pos + inc) & mask) {
            long p0 = pos | op->cval;
            long p1 = p0 | tmask;
            tmp = m[1] * state[p1];
            state[p1] = m[2] * state[p0];
            state[p0] = tmp;
        }
    }
}


void SFX(oracle_serial)(REAL *state_ri, int qubits, const oracle_op *ops, long n_ops, int iterations) {
    cplx *state = (cplx *)state_ri;
    long mem_size = 1L << qubits;
    for (int it = 0; it < iterations; it++) {
        for (long i = 0; i < n_ops; i++) {
            cplx m[4];
            load_matrix(&ops[i], m);
            switch (matrix_type(m)) {
                case DENSE: serial_dense(state, &ops[i], m, mem_size); break;
                case DIAG_PRI: serial_diag(state, &ops[i], m, mem_size); break;
                case DIAG_SEC: serial_antidiag(state, &ops[i], m, mem_size); break;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Region engine: PCpuExecution1 (dgm_par_exec.cpp:82-132).             */
/* ------------------------------------------------------------------ */

typedef struct {
    long region_mask, region_bits, region_count, pos_count, op_end;
} region_plan;

/* compute_region, dgm_par_exec.cpp:38-77 (op_search_end = -1,
 * outer_bound_bits = qubits, parent_mask = -1 as PCpuExecution1 calls it). */
static region_plan compute_region(const oracle_op *ops, long n_ops, long op_start, long coalesced_bits,
                                  long region_bits, long qubits) {
    long count = coalesced_bits;
    long mask = coalesced_bits ? (1L << coalesced_bits) - 1 : 0;
    long i = op_start;
    while (count < region_bits && i < n_ops) {
        if (!((mask >> ops[i].target) & 1)) count++;
        if (count <= region_bits) mask |= (1L << ops[i].target);
        i++;
    }
    while (i < n_ops) {
        if ((mask >> ops[i].target) & 1) i++;
        else break;
    }
    for (long bit = 1; count < region_bits; bit <<= 1) {
        if (bit & ~mask) {
            mask |= bit;
            count++;
        }
    }
    if (count < region_bits) region_bits = count;
    region_plan p;
    p.region_mask = mask;
    p.region_bits = region_bits;
    p.region_count = (1L << (qubits - region_bits)) + 1;
    p.pos_count = 1L << (region_bits - 1);
    p.op_end = i;
    return p;
}

/* PCpuExecution1_0, dgm_par_exec.cpp:138-253 */
static void region_apply(cplx *state, const oracle_op *ops, long start, long end, long pos_count, long region_id,
                         long region_mask, int qubits) {
    for (long i = start; i < end; i++) {
        const oracle_op *op = &ops[i];
        cplx m[4], tmp;
        load_matrix(op, m);
        int type = matrix_type(m);
        long tmask = 1L << op->target;
        long rid = region_id, rmask = region_mask, count = pos_count;
        if (op->cmask) {
            if ((op->cmask & region_id & ~region_mask) != (op->cval & ~region_mask)) continue;
            rid = region_id | op->cval;
            for (int q = 0; q < qubits; q++) {
                long bit = 1L << q;
                if (bit & region_mask & op->cmask) {
                    rmask ^= bit;
                    count /= 2;
                }
            }
        }
        long pos_mask = rmask & ~tmask;
        long inc = ~pos_mask + 1;
        long pos = 0;
        for (long k = 0; k < count; k++) {
            long p0 = pos | rid;
            long p1 = p0 | tmask;
            pos = (pos + inc) & pos_mask;
            switch (type) {
                case DENSE:
                    tmp = m[2] * state[p0] + m[3] * state[p1];
                    state[p0] = m[0] * state[p0] + m[1] * state[p1];
                    state[p1] = tmp;
                    break;
                case DIAG_PRI:
                    tmp = m[3] * state[p1];
                    state[p0] *= m[0];
                    state[p1] = tmp;
                    break;
                default:
                    tmp = m[2] * state[p0];
                    state[p0] = m[1] * state[p1];
                    state[p1] = tmp;
                    break;
            }
        }
    }
}

void SFX(oracle_regions)(REAL *state_ri, int qubits, const oracle_op *ops, long n_ops, int iterations,
                         int threads, int coalesced_bits, int region_bits) {
    cplx *state = (cplx *)state_ri;
    if (region_bits > qubits) region_bits = qubits; /* DGM::validateTuning, dgm_core.cpp:184 */
    if (coalesced_bits > region_bits) coalesced_bits = region_bits;
    for (int it = 0; it < iterations; it++) {
        long op = 0;
        while (op < n_ops) {
            region_plan p = compute_region(ops, n_ops, op, coalesced_bits, region_bits, qubits);
            region_bits = (int)p.region_bits;
            long n_regions = 1L << (qubits - p.region_bits);
            /* Region ids enumerate the bits outside region_mask
             * (next = (id + mask + 1) & ~mask, dgm_par_exec.cpp:107). */
            long outside = ~p.region_mask & ((1L << qubits) - 1);
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
            for (long r = 0; r < n_regions; r++) {
                /* deposit r into the bits of `outside` */
                long id = 0, src = r;
                for (int b = 0; b < qubits && src; b++) {
                    if ((outside >> b) & 1) {
                        id |= (src & 1L) << b;
                        src >>= 1;
                    }
                }
                region_apply(state, ops, op, p.op_end, p.pos_count, id, p.region_mask, qubits);
            }
            op = p.op_end;
        }
    }
}

/* ------------------------------------------------------------------ */
/* FP64 reductions used by the checks.                                  */
/* ------------------------------------------------------------------ */

double SFX(oracle_norm)(const REAL *s, int qubits) {
    long n = 1L << qubits;
    double acc = 0.0;
    for (long i = 0; i < n; i++) acc += (double)s[2 * i] * s[2 * i] + (double)s[2 * i + 1] * s[2 * i + 1];
    return acc;
}

/* Probability that index bit `bit` is 1 (DGM::measure's `one` sum,
 * dgm_core.cpp:79-84, accumulated in FP64). */
double SFX(oracle_prob_one)(const REAL *s, int qubits, int bit) {
    long n = 1L << qubits;
    double acc = 0.0;
    for (long i = 0; i < n; i++)
        if ((i >> bit) & 1) acc += (double)s[2 * i] * s[2 * i] + (double)s[2 * i + 1] * s[2 * i + 1];
    return acc;
}
