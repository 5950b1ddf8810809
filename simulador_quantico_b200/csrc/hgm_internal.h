// Internal declarations shared by the engine's host (C++) and device (CUDA)
// translation units.
#pragma once

#include <cuda_runtime.h>

#include <complex>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "hgm_b200.h"

namespace hgm {

using cplx = std::complex<double>;

// Matrix classes, the reference's PT::matrixType (src/core/common.cpp:33-38)
// by exact zero tests.
enum MatClass : int { MC_DENSE = 0, MC_DIAG = 1, MC_ANTI = 2 };

// One compiled controlled 1-qubit gate (the fields of struct PT the engines
// read, include/core/common.h:57-90).  Matrices are kept in FP64.
struct Op {
    int target = 0;
    uint64_t cmask = 0, cval = 0;
    cplx m[4];
};

MatClass classify(const cplx m[4]);

// ---- errors ---------------------------------------------------------------
void set_error(const char *fmt, ...);
int fail(int code, const char *fmt, ...);

// ---- circuit language ------------------------------------------------------
struct Circuit {
    std::map<std::string, std::vector<cplx>> gates;
    std::vector<Op> ops;
    int qubits = 0;
    // reference-layout PT export (hgm_circuit_ref_pts)
    std::vector<unsigned char> pt_storage;
    std::vector<void *> pt_ptrs;
    std::vector<unsigned char> mat_storage;

    Circuit();
    bool add_gate(const std::string &name, const cplx m[4]);
    int set_function(const std::string &steps, int iterations, bool reset);
};

// ---- kernel-side encodings (shared with kernels.cuh) ----------------------

// Register layouts of a tile (kernels.cuh).  A layout gives every role of
// a thread's view of the tile its local tile bit: thread bits t = 0..4+W
// (lanes 0..4, then warps) at pos[t], register bits q = 0..R-1 at
// pos[5 + W + q].  On the device a layout is a table of LAYOUT_HDR words
// (byte offset in the transpose buffer of each register bit's unit step)
// followed by one word per thread (byte offset of its register 0).
constexpr int MAX_LAYOUT_ROLES = 16;
constexpr int LAYOUT_HDR = 8;
struct Lay {
    int8_t pos[MAX_LAYOUT_ROLES];
};

enum DevKind : int32_t {
    K_DENSE = 0,   // general 2x2
    K_REAL = 1,    // all four entries real
    K_DIAG = 2,    // diag(m00, m11)
    K_PHASE = 3,   // diag(1, m11)
    K_ANTI = 4,    // [[0, m01], [m10, 0]]
    K_SWAP = 5,    // [[0, 1], [1, 0]]
    K_LAYER = 6,   // one uncontrolled dense gate on every register bit; the
                   // R matrices follow in the next R records (bit 0 first)
    K_LAYER_REAL = 7,  // the same with real matrices
    K_PHASE_BLOCK = 8, // diagonal gates with at most one control, combined:
                       // head record (term counts per category in m[] as
                       // bytes, cm_reg bit 0: a 2^R table follows, cv_reg:
                       // active categories), then the term records by
                       // category, then the table
    K_LAYER_SPLIT = 9, // uncontrolled gates R diag(1, p), R real, on the
                       // register bits of the mask (cm_reg): one record per
                       // bit, lowest bit first, with R row-major in m[0..3]
                       // and p in m[4..5]; cv_reg bit b: bit b has a p (a
                       // gate's phase after R follows as a K_PHASE record)
    K_XSET = 10,       // X gates on register bits with at most one control, on
                       // a thread or non-tile bit: tpos entries of 4 bytes
                       // in m[] (target register bit, control kind
                       // XSET_CTRL_*, control bit, control value); each flips
                       // the thread's relabeling mask where its control holds
};
constexpr int XSET_CTRL_NONE = 0, XSET_CTRL_THREAD = 2, XSET_CTRL_GLOBAL = 3;
// entries of one K_XSET record: 4 bytes each in m[]
template <typename Real>
constexpr int xset_entries() {
    return (int)(sizeof(Real) * 8 / 4);
}

// Phase-block term categories (kernels.cuh apply_phase_block): F multiplies
// every register; G[b] the registers whose register bit b is 1, H[b] those
// where it is 0; D[b] a diagonal gate on register bit b (d0 on H[b], d1 on
// G[b]).  Counts are stored in this order: F, G[0..R-1], H[0..R-1], D[0..R-1].
constexpr int PB_MAX_R = 5;
// Terms per phase-block category (the counts are bytes).
constexpr int PB_TERMS = 255;
// Phase-block head: cv_reg bit b (b < R) marks register bit b as having
// G/H/D terms; this bit marks F terms.
constexpr uint32_t PB_F_ACTIVE = 1u << 16;
// Phase-block head flags (cm_reg): a 2^R table follows the terms; the terms
// are compact phase terms (PhaseTerm, several per record) and m[] bytes
// 16..23 hold the index bit of each thread bit (lanes 0..4, warps 5..7).
constexpr uint32_t PB_HAS_TABLE = 1u;
constexpr uint32_t PB_ANGLES = 2u;
// Phase-block head flag (cm_reg, compact terms only): every factor of the
// block is 1 on the registers whose label bit g is 0 -- its only terms are
// G[g] and D[g] terms that add nothing where bit g is 0, and its table is 1
// wherever bit g is 0 -- with g in cm_reg bits PB_GATE_SHIFT.. (the block
// after the QFT's H on register bit g: controlled phases that all involve g).
// Such a block multiplies only half the registers, once each, and always has
// a table (all ones if no term is on register bits only).
constexpr uint32_t PB_GATED = 4u;
constexpr int PB_GATE_SHIFT = 8;


// Target location codes inside a phase: 0..R-1 register bit, 8+q thread bit q
// (lane bits 0..4, warp bits 5..), 64+g a non-tile index bit g.
constexpr int TPOS_THREAD = 8;
constexpr int TPOS_GLOBAL = 64;

template <typename Real>
struct alignas(16) DevOp {
    int32_t kind, tpos;
    uint32_t cm_reg, cv_reg;   // controls on register bits
    uint32_t cm_thr, cv_thr;   // controls on thread bits (lane | warp << 5)
    int32_t tpos2;             // tpos again, so a phase-block term's thread controls and
    uint32_t pad1;             // target come in one 16-byte load
    uint64_t cm_glob, cv_glob; // controls on non-tile index bits
    Real m[8];
};

// A phase-block term whose diagonal entries are pure phases: where its
// control holds (index bit cbit == cval; cbit < 0: no control), it adds a0
// or a1 turns (arguments / 2pi of d0, d1) to the phase of its category, by
// the value of index bit tbit (tbit < 0: a D term, whose category's
// register bit decides).
template <typename Real>
struct PhaseTerm {
    int8_t cbit, cval, tbit;
    int8_t pad[sizeof(Real) - 3];
    Real a0, a1, pad2;
};
// A linear phase term (cbit == PB_LINEAR): many terms of one category whose
// turns are weights w_b on index bits b folded into one.  It adds
// scale * value(ix & mask) turns, where value is the masked index as an
// integer (w_b = scale * 2^b) or, with cval bit 0 set, bit-reversed
// (w_b = scale * 2^-b: brev64(ix & mask) * 2^-63), and only where index bit
// tbit is 1 (tbit < 0: always).  The mask takes the bytes of a0 and a1 (FP32)
// or of a0 (FP64); the scale takes pad2 (FP32) or a1 (FP64).  In a D
// category a linear term adds to the registers whose bit is 1 (its a0 is 0).
// The QFT's controlled phases are such runs: the turns 2^-(t-c+1) of the
// phases on target t from controls c < t are scale 2^-(t+1) times 2^c.
constexpr int8_t PB_LINEAR = -2;
template <typename Real>
constexpr int pb_terms_per_record() {
    return (int)(sizeof(DevOp<Real>) / sizeof(PhaseTerm<Real>));
}

struct DevPhase {
    int32_t layout;          // index into the plan's layout table
    int32_t op_begin, op_end;
    int32_t xwarp;   // 1 if entering this phase needs a cross-warp transpose
};

// Amplitudes a thread keeps in registers, 2^R: R = HGM_F64_REG_BITS for
// FP64 (16 double2 by default) and HGM_F32_REG_BITS for FP32 (32 float2 by
// default).
#ifndef HGM_F32_REG_BITS
#define HGM_F32_REG_BITS 5
#endif
#ifndef HGM_F64_REG_BITS
#define HGM_F64_REG_BITS 4
#endif
// The settings the planner and the tests cover: FP64 4, FP32 4 or 5 (an FP64
// tile of 2^3 registers left the planner with layouts it cannot build).
static_assert(HGM_F64_REG_BITS == 4, "FP64 tiles keep 16 amplitudes a thread");
static_assert(HGM_F32_REG_BITS == 4 || HGM_F32_REG_BITS == 5, "FP32 tiles keep 16 or 32 amplitudes a thread");
constexpr int reg_bits_for(int precision) { return precision == HGM_F64 ? HGM_F64_REG_BITS : HGM_F32_REG_BITS; }
// Register bits of a plan: `requested` (hgm_plan_opts.reg_bits) when valid
// for the precision, -1 when not; requested < 0 picks reg_bits_for.  FP32
// plans may keep 16 amplitudes a thread instead of 32.  That measured faster
// alone for states of at most 20 qubits (Grover, layered and QFT circuits:
// 5-16% with 8 warps a CTA), slower from 22 qubits (35-55%), and slower for
// the serving mix as a whole (303 against 345 circuits/s, with 4 warps a
// CTA), so it is not the default.
inline int plan_reg_bits(int precision, int qubits, int requested) {
    (void)qubits;
    if (precision == HGM_F64) return (requested < 0 || requested == HGM_F64_REG_BITS) ? HGM_F64_REG_BITS : -1;
    if (requested == 4 || requested == 5) return requested;
    return requested < 0 ? HGM_F32_REG_BITS : -1;
}

constexpr int MAX_TILE_BITS = 16;
// Runs of consecutive non-tile index bits: at most one more than tile bits.
constexpr int MAX_FREE_RUNS = MAX_TILE_BITS + 2;

struct PassArgs {
    int32_t n;            // qubits
    int32_t k;            // tile bits = 5 + R + W
    int32_t phase_begin, phase_end;
    int32_t load_layout, store_layout;  // layout table indices
    int32_t flags;        // PASS_* below
    int32_t store_xwarp;  // the transpose into the store layout crosses warps
    int8_t tb[MAX_TILE_BITS];  // local tile bit -> global index bit
    uint64_t tile_mask;
    const DevPhase *phases;
    const void *ops;      // DevOp<Real>*
    double *norm_out;     // PASS_NORM: accumulate sum |a|^2 of stored amplitudes
    const double *scale_in; // PASS_SCALE: multiply loaded amplitudes by 1/sqrt(*scale_in)
    const uint32_t *layouts;  // layout table, LAYOUT_HDR + 2^(5+W) words per layout
    // The non-tile index bits as runs, lowest first: the tile number's next
    // run_len[i] bits go to index bits run_pos[i] .. run_pos[i] + run_len[i] - 1.
    int8_t run_pos[MAX_FREE_RUNS];
    int8_t run_len[MAX_FREE_RUNS];
    int32_t nruns;
    // global index bit of every role of the load and store layouts
    int8_t ld_gbit[MAX_LAYOUT_ROLES];
    int8_t st_gbit[MAX_LAYOUT_ROLES];
};

constexpr int32_t PASS_NORM = 1;
constexpr int32_t PASS_SCALE = 2;

// Small-state path (n < 5 + R): whole state in one CTA's shared memory, ops
// applied one at a time.
template <typename Real>
struct SmallOp {
    int32_t target, kind;
    uint32_t cmask, cval;
    Real m[8];
};

// ---- plan ------------------------------------------------------------------
// Where a plan's device records come from: cudaMalloc/cudaFree by default, or
// an owner's cache (the server recycles them, so that serving makes no
// allocation calls once warm).
struct DevAllocator {
    virtual cudaError_t alloc(void **p, size_t bytes) = 0;
    virtual void free(void *p, size_t bytes) = 0;
    virtual ~DevAllocator() {}
};

struct Plan {
    int precision = HGM_F64;
    int qubits = 0;
    int warp_bits = 0;
    int reg_bits = 5;                 // amplitudes per thread = 2^reg_bits
    bool small = false;               // n < 5 + reg_bits: single-CTA shared-memory path
    std::vector<PassArgs> passes;     // device pointers patched after upload
    std::vector<DevPhase> phases;
    std::vector<Lay> layouts;         // every layout the phases use
    std::vector<unsigned char> ops_bytes;   // DevOp<Real>[] or SmallOp<Real>[]
    int64_t n_small_ops = 0;
    int64_t n_ops = 0, n_transposes = 0;
    // device copies, and their sizes as allocated
    DevAllocator *allocator = nullptr;
    size_t d_bytes[6] = {0, 0, 0, 0, 0, 0};  // ops, phases, layouts, norm, chain scratch, chain passes
    void *d_phases = nullptr;
    void *d_layouts = nullptr;
    void *d_ops = nullptr;
    int renorm_every = 0;
    double *d_norm = nullptr;         // renormalisation scratch (FP32 plans)
    // Chained execution (launch_plan_chain), set up at upload for states of
    // at most CHAIN_MAX_BYTES: the pass records on the device and the
    // scratch (counters, error word, chain_slots renormalisation slots).
    void *d_chain = nullptr;
    void *d_chain_passes = nullptr;
    int64_t chain_slots = 0;
    bool chained = true;              // hgm_plan_opts.chained
    // The plan runs on the pass kernel's lean build: its phase blocks are all
    // compact terms, it has no controlled dense, real or anti-diagonal gate on
    // a register bit and no complex layer (planner, lean_ops).
    bool lean = false;
    // Borrowers (requests of a server, hgm_server_submit_plan) hold a lease;
    // hgm_plan_free on a leased plan only marks it, and the last lease frees
    // it (plan_lease / plan_unlease, engine.cpp).
    int leases = 0;
    bool free_pending = false;
    ~Plan();
};

// States up to this size run their passes chained in one launch (they fit
// in L2 many times over, so a pass lasts a few microseconds and per-pass
// launches would dominate).
constexpr int64_t CHAIN_MAX_BYTES = int64_t(32) << 20;

// Synchronous copy of a state between host and device memory (hostcopy.cpp):
// large copies go through page-locked staging chunks on several threads.
int copy_state(void *dst, const void *src, size_t bytes, bool to_device, void *stream);

// force_small: plan the state for the one-CTA shared-memory path even when
// it is large enough for the register tile (the batched kernel's small tasks).
int build_plan(const std::vector<Op> &ops, int qubits, const hgm_plan_opts &opts, Plan *plan,
               bool force_small = false);
int upload_plan(Plan *plan);
void plan_lease(const Plan *plan);
void plan_unlease(const Plan *plan);

// ---- device state ------------------------------------------------------------
struct State {
    int qubits = 0;
    int precision = HGM_F64;
    void *d = nullptr;
    bool owned = true;   // false: a view into memory another object owns (batch arena, server pool)
    int64_t bytes() const { return (int64_t(1) << qubits) * (precision == HGM_F64 ? 16 : 8); }
};

// ---- launchers (kernels.cu) ----------------------------------------------------
int launch_plan(State *s, const Plan *p, int iterations, void *stream);
// The same in pieces: queues up to max_launches more launches of the plan
// from cursor c (which carries the renormalisation slots across calls).
struct PlanCursor {
    int64_t next = 0;
    int slot = 0;
    bool scale_next = false;
    int scale_slot = 0;
};
int launch_plan_steps(State *s, const Plan *p, int iterations, PlanCursor *c, int64_t max_launches, void *stream);
int64_t plan_launches(const Plan *p, int iterations);
// The whole pass sequence of `iterations` runs of the plan in one persistent
// launch (kernels.cu chain_kernel); only for plans chain_eligible() accepts.
bool chain_eligible(const Plan *p, int iterations);
int launch_plan_chain(State *s, const Plan *p, int iterations, void *stream);
// Device address of the error word the last chained run of p set (nonzero:
// a bounded wait gave up), for an asynchronous copy behind the run.
const void *chain_error_word(const Plan *p);
int launch_set_basis(State *s, int64_t index, void *stream);
int reduce_norm(State *s, double *out, void *stream);
int reduce_prob_one(State *s, int bit, double *out, void *stream);
int collapse(State *s, int bit, int value, double inv_norm, void *stream);
int measure_update(State *s, int bit, int value, double inv_norm, void *stream);
int marginal_argmax(State *s, uint64_t mask, int64_t *arg, double *prob, void *stream);
int marginal_probs(State *s, uint64_t mask, double *host_out, void *stream);
int inner(State *a, State *b, double *re, double *im, void *stream);
int max_abs_diff(State *a, State *b, double *out, void *stream);
int scale_state(State *s, double scale, void *stream);

// Asynchronous FP64 reductions into caller-owned device scratch (used by
// concurrent clients such as the server's slots): partials holds
// 2*REDUCE_SCRATCH_BLOCKS doubles, ibest REDUCE_SCRATCH_BLOCKS indices;
// norm -> out[0]; marginal argmax probability -> out[0], index -> out[1].
constexpr int REDUCE_SCRATCH_BLOCKS = 1184;
int launch_norm_async(State *s, double *partials, double *out, void *stream);
int launch_argmax_async(State *s, uint64_t mask, double *pbest, long long *ibest, double *out, void *stream);

void *default_stream();
void count_launch(int n = 1);

}  // namespace hgm
