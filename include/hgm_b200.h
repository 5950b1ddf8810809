/*
 * hgm_b200.h -- native C-ABI of the B200 state-vector engine (libhgm_b200.so).
 *
 * Plain pointers and sizes only.  Every function returns an int status
 * (HGM_OK == 0) unless noted; hgm_last_error() gives the message of the
 * last failure on the calling thread.
 *
 * Conventions shared with the reference (MMullerdR/simulador_quantico):
 *   - a state of n qubits is 2^n interleaved complex amplitudes (re, im);
 *     index bit b belongs to circuit qubit n-1-b
 *     (docs/01-arquitetura-geral.md, src/core/dgm_core.cpp:72);
 *   - an op is a controlled 1-qubit gate: target index bit, control mask and
 *     value (applied iff (index & mask) == value) and a row-major 2x2 complex
 *     matrix [m00, m01, m10, m11] given as 8 doubles (re, im)
 *     (struct PT, include/core/common.h:57-90; src/core/kernel.cu:109-111).
 *
 * Precision: HGM_F64 states hold complex128, HGM_F32 complex64 (gate
 * matrices are always built in FP64 and cast).
 */
#ifndef HGM_B200_H
#define HGM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HGM_OK 0
#define HGM_ERR_INVALID 1      /* bad argument / malformed circuit */
#define HGM_ERR_CUDA 2         /* CUDA runtime error */
#define HGM_ERR_NOMEM 3        /* device allocation failed / over budget */
#define HGM_ERR_UNSUPPORTED 4  /* feature or size not provided */
#define HGM_ERR_TIMEOUT 5      /* a bounded device wait gave up */
#define HGM_ERR_BUSY 6         /* admission refused (serving) */

#define HGM_F64 0
#define HGM_F32 1

typedef struct hgm_circuit hgm_circuit;
typedef struct hgm_plan hgm_plan;
typedef struct hgm_state hgm_state;

/* ---- runtime ---------------------------------------------------------- */

/* Message of the last failed call on this thread ("" if none). */
const char *hgm_last_error(void);
/* Initialises the CUDA context on `device` (setDevice, src/core/kernel.cu:31-33).
 * Sets CUDA_DEVICE_MAX_CONNECTIONS=32 first unless the environment has it
 * (one hardware queue per server slot; effective only before the process
 * creates its CUDA context). */
int hgm_init(int device);
/* Blocks until all work queued by this library has finished. */
int hgm_synchronize(void);
/* Free / total device memory in bytes. */
int hgm_mem_info(int64_t *free_bytes, int64_t *total_bytes);
/* Page-locked host memory (cudaMallocHost), for asynchronous copies. */
int hgm_pinned_alloc(int64_t bytes, void **out);
void hgm_pinned_free(void *p);
/* Number of kernel launches issued by this library since load. */
int64_t hgm_kernel_launches(void);

/* ---- circuits: host mirror of the DGM circuit language ------------------ */
/* The circuit language of docs/02-linguagem-de-circuitos.md: steps separated
 * by ';', one token per qubit separated by ','; tokens ID, a gate name,
 * ControlN(v), TargetN(gate).  Parsed exactly as DGM::setFunction /
 * genGroups / genPTs (src/core/dgm_parser.cpp:29-169). */

hgm_circuit *hgm_circuit_new(void);
void hgm_circuit_free(hgm_circuit *c);
/* Gates::addGate (src/core/gates.cpp:42-60): registers a 2x2 matrix under
 * `name`; returns 1 if added, 0 if the name already exists (never
 * overwrites), <0 on error. */
int hgm_circuit_add_gate(hgm_circuit *c, const char *name, const double m[8]);
/* DGM::setFunction(string, iterations, reset) (dgm_parser.cpp:29-66). */
int hgm_circuit_set_function(hgm_circuit *c, const char *steps, int iterations, int reset);
/* Appends one op directly (no string). */
int hgm_circuit_append_op(hgm_circuit *c, int target, int64_t cmask, int64_t cval, const double m[8]);
/* Width of the last parsed step (DGM::qubits after genGroups). */
int hgm_circuit_qubits(const hgm_circuit *c);
int64_t hgm_circuit_num_ops(const hgm_circuit *c);
/* Copies the compiled op list out (arrays of num_ops entries; m: 8 per op). */
int hgm_circuit_get_ops(const hgm_circuit *c, int32_t *target, int64_t *cmask, int64_t *cval, double *m);
/* Exposes the op list as a NULL-terminated array of reference-layout PTs
 * (struct hgm_ref_pt of hgm_dropin.h) whose matrices have the given
 * precision; owned by the circuit, valid until the next change. */
void *hgm_circuit_ref_pts(hgm_circuit *c, int precision);

/* ---- plans: op list -> state passes ------------------------------------ */

typedef struct hgm_plan_opts {
    int precision;   /* HGM_F64 / HGM_F32 */
    int warp_bits;   /* tile = 2^(10+warp_bits) amplitudes; -1 = default */
    int low_bits;    /* contiguous low index bits kept in every tile; -1 = default */
    int fuse;        /* 1 = fuse adjacent gates on the same target and
                        controls; 2 = the same, except a pure phase next to a
                        real gate (kept apart: the real gate takes the
                        cheaper real form, the phase joins a phase block);
                        0 = no fusion */
    int window;      /* scheduling look-ahead in ops; <=0 = default */
    int renorm_every;/* FP32: rescale to unit norm every k passes (0 = never) */
    int chained;     /* 1 (default): a state of at most 32 MiB runs all its passes
                        in one persistent launch; 0: one launch per pass */
    int split_layers;/* 1 (default): an uncontrolled dense gate of a layer
                        whose matrix is s diag(1,q) R diag(1,p) with R real and
                        |s| = |p| = |q| = 1 (every unitary is) runs as phase,
                        real gate, phase, and the scalars s of all such gates
                        are applied once at the end of the plan; 0: every dense
                        gate runs as a complex matrix */
    int reg_bits;    /* amplitudes a thread keeps in registers = 2^reg_bits:
                        FP64 4; FP32 4 or 5; -1 = default (FP64 4, FP32 5) */
} hgm_plan_opts;

void hgm_plan_default_opts(hgm_plan_opts *o, int precision);
int hgm_plan_create(const hgm_circuit *c, int qubits, const hgm_plan_opts *opts, hgm_plan **out);
/* Same, from a reference-layout NULL-terminated PT list (hgm_ref_pt**). */
int hgm_plan_create_from_ref_pts(void *const *pts, int pt_precision, int qubits, const hgm_plan_opts *opts,
                                 hgm_plan **out);
/* Waits for the work queued on the device, then frees the plan: a plan may be
 * freed right after the executions that use it are queued.  A plan that
 * requests submitted with hgm_server_submit_plan still use is freed when the
 * last of them is done. */
void hgm_plan_free(hgm_plan *p);
/* Plan statistics: ops after fusion, passes, phases, transposes. */
int hgm_plan_stats(const hgm_plan *p, int64_t *n_ops, int64_t *n_passes, int64_t *n_phases, int64_t *n_transposes);
/* Copies the plan's device records to the GPU now instead of at its first
 * execution or submission (so that a timed or latency-critical section does
 * not pay for the allocation and copy). */
int hgm_plan_upload(hgm_plan *p);

/* Read-only view of a plan's host-side encoding (for inspection and the
 * CPU emulation test): per-pass kernel arguments (struct PassArgs), register
 * phases (struct DevPhase) and encoded gates (DevOp or SmallOp records), as
 * laid out in simulador_quantico_b200/csrc/hgm_internal.h. */
int hgm_plan_export(const hgm_plan *p, const void **passes, int64_t *n_passes, const void **phases,
                    int64_t *n_phases, const void **ops, int64_t *ops_bytes, int *warp_bits, int *small);
/* The plan's register layouts (struct Lay: 16 int8 local tile bits per
 * layout, thread bits first, then register bits), for the same emulation. */
int hgm_plan_layouts(const hgm_plan *p, const int8_t **pos, int64_t *n_layouts);

/* ---- device-resident states -------------------------------------------- */

int hgm_state_create(int qubits, int precision, hgm_state **out);
/* Waits for the work queued on the device, then frees the state. */
void hgm_state_free(hgm_state *s);
int hgm_state_qubits(const hgm_state *s);
int hgm_state_precision(const hgm_state *s);
void *hgm_state_device_ptr(hgm_state *s);
/* |index> (DGM::setMemoryValue, src/core/dgm_core.cpp:63-65). */
int hgm_state_set_basis(hgm_state *s, int64_t index);
/* Host <-> device copies of the whole state (bytes = 2^n * amplitude size). */
int hgm_state_upload(hgm_state *s, const void *host, int64_t bytes);
int hgm_state_download(const hgm_state *s, void *host, int64_t bytes);

/* ---- execution ---------------------------------------------------------- */

/* Applies the plan `iterations` times on `stream` (0 = the library stream).
 * A state of at most 32 MiB (22 qubits FP32, 21 FP64) runs every pass in
 * one persistent launch instead of one launch per pass; that launch's
 * passes wait on each other with a bounded wait (hgm_plan_status).  The
 * chained run's counters and an FP32 plan's renormalisation slots belong to
 * the plan: executions of one plan must not overlap on the device. */
int hgm_execute(hgm_state *s, const hgm_plan *p, int iterations, void *stream);
/* After the plan's executions have been queued: waits for the device, then
 * HGM_ERR_TIMEOUT if the last chained execution of the plan gave up a wait
 * (its result is then not valid), else HGM_OK. */
int hgm_plan_status(const hgm_plan *p);

/* ---- device-resident measurement (FP64 reductions) ---------------------- */

/* sum |a|^2 */
int hgm_norm(hgm_state *s, double *out);
/* Probability that index bit `bit` is 1 (DGM::measure's sums, dgm_core.cpp:79-84). */
int hgm_prob_one(hgm_state *s, int bit, double *out);
/* DGM::measure(qubit) (dgm_core.cpp:69-125) on the device, with the uniform
 * sample in [0, 1) supplied by the caller: outcome 0 if P(0) > sample else 1.
 * As in the reference, the measured branch is renormalised and moved to the
 * qubit's |0> half and the |1> half is cleared, so the qubit is left in |0>
 * whichever value was read (dgm_core.cpp:115-122).  Returns the outcome and
 * its probability. */
int hgm_measure_qubit(hgm_state *s, int qubit, double sample, int *outcome, double *prob);
/* DGM::colapse(qubit, value) (dgm_core.cpp:129-146): keeps the amplitudes in
 * which `qubit` has `value`, renormalised, and clears the others; returns the
 * probability that was collapsed onto (the reference prints it). */
int hgm_collapse_qubit(hgm_state *s, int qubit, int value, double *prob);
/* DGM::measure(vector<int>) (dgm_core.cpp:150-162): the probabilities of every
 * value of the index bits in `mask`, summed over the other bits, without
 * collapsing; out[x] for x = 0 .. 2^popcount(mask)-1, where bit j of x is the
 * j-th lowest bit of `mask` (the reference keys the same sums by
 * index & mask).  count must be 2^popcount(mask), at most 2^26. */
int hgm_marginal_probs(hgm_state *s, uint64_t mask, double *out, int64_t count);
/* Marginal distribution over the index bits in `mask`: argmax of
 * sum over the other bits of |a|^2 (ties -> lowest index). */
int hgm_marginal_argmax(hgm_state *s, uint64_t mask, int64_t *arg, double *prob);
/* <a|b> accumulated in FP64 (a, b may differ in precision, same qubits). */
int hgm_inner(hgm_state *a, hgm_state *b, double *re, double *im);
/* max_i |a_i - b_i| */
int hgm_max_abs_diff(hgm_state *a, hgm_state *b, double *out);
/* Multiplies every amplitude by `scale`. */
int hgm_scale(hgm_state *s, double scale);

/* Allocation-free FP64 norm: sum |a|^2 of the device state `d_state`
 * (2^qubits amplitudes of the given precision), written to the one device
 * double at `d_out` (8 bytes; nothing after it is touched), queued on
 * `stream`.  No counterpart in the reference.  For callers that cannot
 * allocate device memory (code inside a framework that owns every
 * allocation and hands this library only its buffers, or code running while
 * another thread captures a CUDA graph, where an allocation would break the
 * capture): it calls no cudaMalloc, cudaFree or allocating routine and keeps
 * its partial sums in an 18.5 KiB device array that every GPU loading this
 * library holds until exit.  Limit: 1..34 qubits, the engine's state range
 * (HGM_ERR_UNSUPPORTED beyond; the array itself fits any size, the grid
 * being capped at its 1184 partials).  All calls share that array: calls
 * that overlap on the GPU race and must be serialised.  The first call on a
 * device looks the array's address up (make it before any stream capture).
 * stream NULL is the legacy default stream, which synchronises with every
 * blocking stream: while another thread captures on a blocking stream, pass
 * a stream created with cudaStreamNonBlocking instead. */
int hgm_norm_noalloc(const void *d_state, int qubits, int precision, double *d_out, void *stream);

/* ---- batched mode --------------------------------------------------------- */
/* Many independent circuits of uneven size run by one persistent kernel that
 * a CUDA graph replays: hgm_batch_add the circuits, hgm_batch_finalize
 * (plans every circuit for the same register tile of 2^(5+R+warp_bits)
 * amplitudes, lays the states out in one device arena, captures the graph),
 * then hgm_batch_run as often as needed.  Each run resets every state to its
 * initial basis index and applies its circuit. */

typedef struct hgm_batch hgm_batch;
int hgm_batch_create(int precision, int warp_bits, hgm_batch **out);
void hgm_batch_free(hgm_batch *b);
/* Adds a circuit on `qubits` qubits starting from |init_index>; returns its job index. */
int hgm_batch_add(hgm_batch *b, const hgm_circuit *c, int qubits, int64_t init_index, int *job);
int hgm_batch_finalize(hgm_batch *b);
/* Launches the graph on `stream` (0 = library stream); asynchronous. */
int hgm_batch_run(hgm_batch *b, void *stream);
/* Autotuner: re-plans the batch for every tile size (warp_bits 0..3) and
 * every count of always-resident low index bits (3..5), times two graph
 * replays of each, and leaves the batch finalized with the fastest; reports
 * the choice and its time per run (ms). */
int hgm_batch_autotune(hgm_batch *b, void *stream, int *warp_bits, int *low_bits, double *ms);
/* Sets every job's initial basis index for the next runs (an asynchronous
 * copy of njobs int64 values on `stream`; pinned memory keeps it so). */
int hgm_batch_set_inputs(hgm_batch *b, const int64_t *init_index, void *stream);
/* Copies every job's state (the arena: jobs back to back in job order, each
 * 2^n amplitudes) to `host` (exactly the arena's bytes; asynchronous on
 * `stream` when `host` is pinned). */
int hgm_batch_download(hgm_batch *b, void *host, int64_t bytes, void *stream);
/* After a run has completed: HGM_ERR_TIMEOUT if a tile gave up waiting. */
int hgm_batch_check(hgm_batch *b);
/* Fault injection for tests, made on the host: from the next run, `task`
 * (an index into the finalized batch's task table; it must have a
 * dependency) waits for one completion more than its dependency can give,
 * and every dependency wait gives up after wait_ns instead of 2 s, so the
 * run ends with HGM_ERR_TIMEOUT from hgm_batch_check.  task < 0 restores the
 * normal table and limit.  Waits for earlier runs first. */
int hgm_batch_inject_stall(hgm_batch *b, int task, int64_t wait_ns);
/* pass_bytes: the algorithmic bytes of one run, a read and a write of a
 * state per pass (per task). */
int hgm_batch_size(const hgm_batch *b, int *jobs, int64_t *tasks, int64_t *items, int64_t *arena_bytes,
                   int64_t *pass_bytes);
/* A view of one job's state (owned by the batch; hgm_state_free ignores it). */
hgm_state *hgm_batch_state(hgm_batch *b, int job);

/* ---- serving mode --------------------------------------------------------- */
/* Continuous batching: circuits are submitted at any time and admitted, in
 * arrival order, while one of max_inflight slots is free and their state
 * bytes (16*2^n FP64, 8*2^n FP32) fit budget_bytes; admitted circuits run
 * concurrently, each on its own stream with a stream-ordered state
 * allocation; every result reports its FP64 norm, the marginal argmax over
 * result_mask (if non-zero) and its latency. */

typedef struct hgm_server hgm_server;
typedef struct hgm_server_opts {
    int precision;         /* HGM_F64 / HGM_F32 */
    int64_t budget_bytes;  /* HBM admission budget for resident states */
    int max_inflight;      /* concurrent requests (streams) */
    int keep_states;       /* 1: finished states stay on the device until hgm_server_release */
    int warp_bits;         /* tile size, -1 = default */
    int order;             /* HGM_ORDER_ARRIVAL: queued requests are admitted in
                              arrival order; HGM_ORDER_WORK_FIRST: the queued
                              request with the most work (state bytes x passes)
                              that fits the budget goes first */
} hgm_server_opts;
#define HGM_ORDER_ARRIVAL 0
#define HGM_ORDER_WORK_FIRST 1

typedef struct hgm_result {
    int64_t id;
    int status;            /* HGM_OK or an error code */
    int qubits;
    double latency_s;      /* submit -> result available */
    double queue_s;        /* submit -> admitted */
    double exec_s;         /* admitted -> result available */
    double norm;           /* sum |a|^2, FP64 */
    int64_t argmax;        /* marginal argmax over result_mask, -1 if not asked */
    double pmax;           /* its probability */
} hgm_result;

void hgm_server_default_opts(hgm_server_opts *o, int precision);
int hgm_server_create(const hgm_server_opts *opts, hgm_server **out);
void hgm_server_free(hgm_server *s);
/* Copies the circuit and queues it; planner threads plan and upload it while
 * earlier requests run (a planning failure comes back as the result's
 * status).  HGM_ERR_BUSY if its state can never fit the budget. */
int hgm_server_submit(hgm_server *s, const hgm_circuit *c, int qubits, int64_t init_index, uint64_t result_mask,
                      int64_t *id);
/* Queues an already built plan (hgm_plan_create, the server's precision):
 * the request's work is then all on the device.  The plan is uploaded here
 * if it has not run yet.  It is borrowed: it must stay alive, and not run
 * elsewhere, until this request's result has been polled (its
 * renormalisation scratch belongs to the plan). */
int hgm_server_submit_plan(hgm_server *s, const hgm_plan *p, int64_t init_index, uint64_t result_mask, int64_t *id);
/* Moves up to `max` finished results into `out` (waiting up to wait_ms for
 * the first); *n = how many. */
int hgm_server_poll(hgm_server *s, hgm_result *out, int max, int *n, int wait_ms);
int hgm_server_pending(hgm_server *s, int *queued, int *inflight, int64_t *bytes_in_use);
/* With keep_states: a view of a finished request's state, valid until release. */
hgm_state *hgm_server_result_state(hgm_server *s, int64_t id);
int hgm_server_release(hgm_server *s, int64_t id);

/* ---- timing (CUDA events on the library stream) ------------------------- */

/* Records an event pair around everything queued between start and stop. */
int hgm_timer_start(void);
int hgm_timer_stop(double *ms);

#ifdef __cplusplus
}
#endif
#endif /* HGM_B200_H */
