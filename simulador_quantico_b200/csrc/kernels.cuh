// Device code of the state-vector engine (sm_100a).
//
// Pass kernel ("register tile" design)
// ------------------------------------
// One CTA owns a tile of 2^K amplitudes, K = 5 + R + W: every thread keeps
// NR = 2^R amplitudes in registers (R = 5 for FP32, 4 for FP64), a warp
// holds 2^(5+R) and the CTA 2^W warps.  The tile is the set of state
// indices that agree on every index bit outside the pass's K tile bits;
// local tile bit q is index bit tb[q].  Which local bits are the lane,
// warp and register bits of a thread is the current phase's layout, a table
// the planner builds (struct Lay): any R local bits can be the register bits.
//
// A gate whose target is a register bit of the current layout is applied
// entirely in registers.  Switching layout is a transpose through shared
// memory; when both layouts keep the warp bits in place it stays inside
// each warp (__syncwarp), otherwise it crosses warps (__syncthreads).  The
// load and store layouts put thread bits 0..low_bits-1 on the lowest index
// bits of the state, so each warp instruction moves whole 128-byte runs.
// Shared memory is padded (pad_slot below); the planner only builds layouts
// whose accesses are free of bank conflicts under that padding.
//
// State loads and stores bypass L1 (ld/st .cg): every amplitude is touched
// once per pass, and a tile written by one CTA may be read by another CTA of
// the same persistent kernel in the next pass, which L2 keeps coherent.
//
// The state is read once and written once per pass (the reference's
// "load a tile, apply the whole gate batch, write back once",
// src/core/kernel.cu:68-128), so a pass moves 2*S bytes of HBM traffic.
#pragma once

#include <cuda_runtime.h>

#include "hgm_internal.h"

namespace hgm {

// Register budget per thread.  The FP32 tile (32 float2) and the FP64 tile
// (16 double2) both hold 64 data registers.  128 lets 4 CTAs of 4 warps share
// an SM; the pass kernel is latency-bound, and the fourth CTA outweighs the
// spills the cap brings (26-qubit layered passes: FP64 -13%, FP32 -2%, QFT
// -12% against a 168-register cap with 3 CTAs per SM).
#ifndef HGM_MAXREG_F32
#define HGM_MAXREG_F32 128
#endif
#ifndef HGM_MAXREG_F64
#define HGM_MAXREG_F64 128
#endif
// Shared-memory carveout for the pass kernels, in percent (-1: driver's
// choice).  The L1 left over holds the loads in flight; forcing the maximum
// shared carveout measured 30% slower streaming passes.
#ifndef HGM_SMEM_CARVEOUT
#define HGM_SMEM_CARVEOUT -1
#endif
template <typename Real, int R>
constexpr int pass_max_regs() {
    return sizeof(Real) == 8 ? HGM_MAXREG_F64 : HGM_MAXREG_F32;
}

template <typename Real>
struct V2;
template <>
struct V2<double> {
    using T = double2;
};
template <>
struct V2<float> {
    using T = float2;
};

// Shared-memory slot of local index j in a transpose: j + (j >> R).  The
// padding keeps every layout's warp accesses free of bank conflicts (a lane
// stride of 2^R elements becomes 2^R + 1) and, unlike an XOR swizzle, it is
// additive over a layout's disjoint lane/warp and register bits, so the slot
// of register r is the thread's base slot plus r times a constant.
template <int R>
__device__ __forceinline__ uint32_t pad_slot(uint32_t j) {
    return j + (j >> R);
}

// Shared memory of one tile's transposes, in amplitudes.
template <int R, int W>
__host__ __device__ constexpr int tile_smem_elems() {
    return (1 << (5 + R + W)) + (1 << (5 + W));
}

// Offset (in amplitudes) of a thread's register-0 amplitude and the R
// register-bit strides in the state, for a layout given by the global index
// bit of each role (thread bits 0..4+W, then register bits).  Every lookup
// uses a constant index into the kernel parameters (a runtime index would
// copy them to local memory).
template <int R, int W>
__device__ __forceinline__ void thread_geometry(const int8_t (&gb)[MAX_LAYOUT_ROLES], uint32_t thr, uint64_t &off,
                                                uint64_t (&rs)[R]) {
    off = 0;
#pragma unroll
    for (int t = 0; t < 5 + W; t++) off |= (uint64_t)((thr >> t) & 1) << gb[t];
#pragma unroll
    for (int q = 0; q < R; q++) rs[q] = (uint64_t)1 << gb[5 + W + q];
}

template <int R, int r>
__device__ __forceinline__ uint64_t reg_offset(const uint64_t (&rs)[R]) {
    uint64_t o = 0;
#pragma unroll
    for (int q = 0; q < R; q++)
        if (r & (1 << q)) o += rs[q];
    return o;
}

template <int r>
struct Unroll {
    template <typename F>
    __device__ __forceinline__ static void run(F &f) {
        Unroll<r - 1>::run(f);
        f.template go<r - 1>();
    }
};
template <>
struct Unroll<0> {
    template <typename F>
    __device__ __forceinline__ static void run(F &) {}
};

template <typename A2, int R>
struct LoadF {
    A2 (&a)[1 << R];
    const A2 *__restrict__ p;
    const uint64_t (&rs)[R];
    template <int r>
    __device__ __forceinline__ void go() {
        a[r] = __ldcg(p + reg_offset<R, r>(rs));
    }
};
// Register r goes to element idx ^ offset(r): idx already carries the
// offset of the relabeling mask (the offsets are disjoint bits, so
// offset(r ^ xr) = offset(r) ^ offset(xr)).
template <typename A2, int R>
struct StoreF {
    const A2 (&a)[1 << R];
    A2 *__restrict__ p;
    uint64_t idx;
    const uint64_t (&rs)[R];
    template <int r>
    __device__ __forceinline__ void go() {
        __stcg(p + (idx ^ reg_offset<R, r>(rs)), a[r]);
    }
};

// ---- in-place amplitude updates --------------------------------------------
// Every update of a register amplitude goes through these inline-PTX
// primitives.  Their amplitude operands are tied ("+"), so each result is
// written into the register that held the input and the amplitudes keep their
// registers from one gate to the next.  Written as plain expressions, the
// compiler left each result in a fresh register and copied it back wherever
// the op loop's dispatch paths merge; those copies outnumbered the
// floating-point instructions of the pass kernel.  Negated coefficients come
// in as operands (PTX fma has no negated-operand form).
#define HGM_INPLACE_PRIMITIVES(REAL, SFX, C)                                                                      \
    /* (x, y) <- M (x, y), complex M = m[0..7] (row-major re/im), n_k = -m_k */                                 \
    __device__ __forceinline__ void ip_dense(REAL &xr, REAL &xi, REAL &yr, REAL &yi, const REAL(&m)[8], REAL n1, \
                                             REAL n3, REAL n5, REAL n7) {                                        \
        asm("{\n\t.reg ." SFX " t0, t1, t2, t3;\n\t"                                                              \
            "mul.rn." SFX " t0, %4, %0;\n\tmul.rn." SFX " t1, %4, %1;\n\t"                                          \
            "mul.rn." SFX " t2, %8, %0;\n\tmul.rn." SFX " t3, %8, %1;\n\t"                                          \
            "fma.rn." SFX " t0, %12, %1, t0;\n\tfma.rn." SFX " t1, %5, %0, t1;\n\t"                                 \
            "fma.rn." SFX " t2, %14, %1, t2;\n\tfma.rn." SFX " t3, %9, %0, t3;\n\t"                                 \
            "fma.rn." SFX " t0, %6, %2, t0;\n\tfma.rn." SFX " t1, %7, %2, t1;\n\t"                                  \
            "fma.rn." SFX " t2, %10, %2, t2;\n\tfma.rn." SFX " t3, %11, %2, t3;\n\t"                                \
            "fma.rn." SFX " %0, %13, %3, t0;\n\tfma.rn." SFX " %1, %6, %3, t1;\n\t"                                 \
            "fma.rn." SFX " %2, %15, %3, t2;\n\tfma.rn." SFX " %3, %10, %3, t3;\n\t}"                               \
            : "+" C(xr), "+" C(xi), "+" C(yr), "+" C(yi)                                                         \
            : C(m[0]), C(m[1]), C(m[2]), C(m[3]), C(m[4]), C(m[5]), C(m[6]), C(m[7]), C(n1), C(n3), C(n5),      \
              C(n7));                                                                                            \
    }                                                                                                            \
    /* (x, y) <- M (x, y), real M = (m00, m01, m10, m11) */                                                      \
    __device__ __forceinline__ void ip_real(REAL &xr, REAL &xi, REAL &yr, REAL &yi, REAL m00, REAL m01,         \
                                            REAL m10, REAL m11) {                                                \
        asm("{\n\t.reg ." SFX " t0, t1, t2, t3;\n\t"                                                              \
            "mul.rn." SFX " t0, %4, %0;\n\tmul.rn." SFX " t1, %6, %0;\n\t"                                          \
            "mul.rn." SFX " t2, %4, %1;\n\tmul.rn." SFX " t3, %6, %1;\n\t"                                          \
            "fma.rn." SFX " %0, %5, %2, t0;\n\tfma.rn." SFX " %2, %7, %2, t1;\n\t"                                  \
            "fma.rn." SFX " %1, %5, %3, t2;\n\tfma.rn." SFX " %3, %7, %3, t3;\n\t}"                                 \
            : "+" C(xr), "+" C(xi), "+" C(yr), "+" C(yi)                                                         \
            : C(m00), C(m01), C(m10), C(m11));                                                                   \
    }                                                                                                            \
    /* x <- x * (fr + i fi), nfi = -fi */                                                                        \
    __device__ __forceinline__ void ip_cmul(REAL &xr, REAL &xi, REAL fr, REAL fi, REAL nfi) {                  \
        asm("{\n\t.reg ." SFX " t0, t1;\n\t"                                                                      \
            "mul.rn." SFX " t0, %2, %0;\n\tmul.rn." SFX " t1, %3, %0;\n\t"                                          \
            "fma.rn." SFX " %0, %4, %1, t0;\n\tfma.rn." SFX " %1, %2, %1, t1;\n\t}"                                 \
            : "+" C(xr), "+" C(xi)                                                                               \
            : C(fr), C(fi), C(nfi));                                                                             \
    }
HGM_INPLACE_PRIMITIVES(double, "f64", "d")
HGM_INPLACE_PRIMITIVES(float, "f32", "f")
#undef HGM_INPLACE_PRIMITIVES

// amplitude a <- a * f (complex factor f)
template <typename A2>
__device__ __forceinline__ void ip_cmul2(A2 &a, A2 f) {
    ip_cmul(a.x, a.y, f.x, f.y, -f.y);
}

// ---- gate application on register bits -----------------------------------

template <typename Real, typename A2>
__device__ __forceinline__ A2 cmul(A2 a, Real mr, Real mi) {
    A2 o;
    o.x = a.x * mr - a.y * mi;
    o.y = a.x * mi + a.y * mr;
    return o;
}

// Each body handles the NR/2 register pairs (or NR registers) of one target
// bit.  Without register-bit controls (CTRL = false, the common case) the
// body is one basic block, so the FMAs of all pairs interleave; with
// controls (CTRL = true) each pair is guarded by its own branch, which keeps
// that rarer variant's register footprint small.
#define HGM_PAIR_GUARD(r) \
    if (CTRL && (((uint32_t)(r) & cm) != cv)) continue;

template <typename Real, typename A2, int R, int T, bool CTRL>
__device__ __forceinline__ void reg_dense(A2 (&a)[1 << R], const Real (&m)[8], uint32_t cm, uint32_t cv) {
    const Real n1 = -m[1], n3 = -m[3], n5 = -m[5], n7 = -m[7];
#pragma unroll
    for (int r = 0; r < (1 << R); r++) {
        if (r & (1 << T)) continue;
        const int r1 = r | (1 << T);
        HGM_PAIR_GUARD(r)
        ip_dense(a[r].x, a[r].y, a[r1].x, a[r1].y, m, n1, n3, n5, n7);
    }
}

// FP32 real 2x2 on packed (re, im) pairs: one f32x2 multiply and one f32x2
// fused multiply-add per output amplitude instead of two of each (the same
// IEEE operations per component, so the results are bit-identical); the
// coefficients come in duplicated, (m, m), built once per gate.
__device__ __forceinline__ void ip_real_x2(float &xr, float &xi, float &yr, float &yi, unsigned long long c00,
                                           unsigned long long c01, unsigned long long c10, unsigned long long c11) {
    asm("{\n\t.reg .b64 X, Y, P, Q;\n\t"
        "mov.b64 X, {%0, %1};\n\tmov.b64 Y, {%2, %3};\n\t"
        "mul.rn.f32x2 P, %4, X;\n\tmul.rn.f32x2 Q, %6, X;\n\t"
        "fma.rn.f32x2 P, %5, Y, P;\n\tfma.rn.f32x2 Q, %7, Y, Q;\n\t"
        "mov.b64 {%0, %1}, P;\n\tmov.b64 {%2, %3}, Q;\n\t}"
        : "+f"(xr), "+f"(xi), "+f"(yr), "+f"(yi)
        : "l"(c00), "l"(c01), "l"(c10), "l"(c11));
}
__device__ __forceinline__ unsigned long long dup_f32(float v) {
    unsigned long long d;
    asm("mov.b64 %0, {%1, %1};" : "=l"(d) : "f"(v));
    return d;
}

template <typename Real, typename A2, int R, int T, bool CTRL>
__device__ __forceinline__ void reg_real(A2 (&a)[1 << R], const Real (&m)[8], uint32_t cm, uint32_t cv) {
    if constexpr (sizeof(Real) == 4) {
        const unsigned long long c00 = dup_f32(m[0]), c01 = dup_f32(m[2]), c10 = dup_f32(m[4]), c11 = dup_f32(m[6]);
#pragma unroll
        for (int r = 0; r < (1 << R); r++) {
            if (r & (1 << T)) continue;
            const int r1 = r | (1 << T);
            HGM_PAIR_GUARD(r)
            ip_real_x2(a[r].x, a[r].y, a[r1].x, a[r1].y, c00, c01, c10, c11);
        }
    } else {
#pragma unroll
        for (int r = 0; r < (1 << R); r++) {
            if (r & (1 << T)) continue;
            const int r1 = r | (1 << T);
            HGM_PAIR_GUARD(r)
            ip_real(a[r].x, a[r].y, a[r1].x, a[r1].y, m[0], m[2], m[4], m[6]);
        }
    }
}

template <typename Real, typename A2, int R, int T, bool CTRL>
__device__ __forceinline__ void reg_diag(A2 (&a)[1 << R], const Real (&m)[8], uint32_t cm, uint32_t cv) {
    const Real n1 = -m[1], n7 = -m[7];
#pragma unroll
    for (int r = 0; r < (1 << R); r++) {
        HGM_PAIR_GUARD(r)
        if (r & (1 << T)) ip_cmul(a[r].x, a[r].y, m[6], m[7], n7);
        else ip_cmul(a[r].x, a[r].y, m[0], m[1], n1);
    }
}

template <typename Real, typename A2, int R, int T, bool CTRL>
__device__ __forceinline__ void reg_phase(A2 (&a)[1 << R], const Real (&m)[8], uint32_t cm, uint32_t cv) {
    const Real n7 = -m[7];
#pragma unroll
    for (int r = 0; r < (1 << R); r++) {
        if (!(r & (1 << T))) continue;
        HGM_PAIR_GUARD(r)
        ip_cmul(a[r].x, a[r].y, m[6], m[7], n7);
    }
}

template <typename Real, typename A2, int R, int T, bool CTRL>
__device__ __forceinline__ void reg_anti(A2 (&a)[1 << R], const Real (&m)[8], uint32_t cm, uint32_t cv) {
#pragma unroll
    for (int r = 0; r < (1 << R); r++) {
        if (r & (1 << T)) continue;
        const int r1 = r | (1 << T);
        HGM_PAIR_GUARD(r)
        const A2 x = a[r], y = a[r1];
        a[r] = cmul<Real>(y, m[2], m[3]);
        a[r1] = cmul<Real>(x, m[4], m[5]);
    }
}

// Controlled swaps select instead of branching: two selects per component
// are cheaper than a branch per pair.
template <typename A2, int R, int T, bool CTRL>
__device__ __forceinline__ void reg_swap(A2 (&a)[1 << R], uint32_t cm, uint32_t cv) {
#pragma unroll
    for (int r = 0; r < (1 << R); r++) {
        if (r & (1 << T)) continue;
        const int r1 = r | (1 << T);
        const A2 x = a[r], y = a[r1];
        if (CTRL) {
            const bool p = ((uint32_t)r & cm) == cv;
            a[r].x = p ? y.x : x.x;
            a[r].y = p ? y.y : x.y;
            a[r1].x = p ? x.x : y.x;
            a[r1].y = p ? x.y : y.y;
        } else {
            a[r] = y;
            a[r1] = x;
        }
    }
}

// Diagonal gate whose target bit is not a register bit: the factor is the
// same for all of a thread's registers that satisfy the register controls.
template <typename Real, typename A2, int R, bool CTRL>
__device__ __forceinline__ void reg_scale(A2 (&a)[1 << R], Real fr, Real fi, uint32_t cm, uint32_t cv) {
    const Real nfi = -fi;
#pragma unroll
    for (int r = 0; r < (1 << R); r++) {
        HGM_PAIR_GUARD(r)
        ip_cmul(a[r].x, a[r].y, fr, fi, nfi);
    }
}

// Kind dispatch as a chain of independent bit tests (not a switch): each
// body updates the registers in place and merges with the path that skips
// it, the shape under which the registers keep their places (a switch here
// became a jump table and cost a hundred register copies per gate).
template <typename Real>
__device__ __forceinline__ void load_matrix(const Real *__restrict__ src, Real (&m)[8]);
template <typename Real>
__device__ __forceinline__ void load_matrix_flip(const Real *__restrict__ src, Real (&m)[8], bool flip);
template <typename Real, typename A2>
__device__ __forceinline__ A2 load_c(const Real *__restrict__ p);

// LEAN: the pass kernel's lean build (plans without controlled dense, real
// or anti-diagonal gates on register bits; Plan::lean) leaves those bodies out.
template <typename Real, typename A2, int R, int T, bool CTRL, bool LEAN>
__device__ __forceinline__ void reg_kind_c(uint32_t kbit, A2 (&a)[1 << R], const Real *__restrict__ mp, uint32_t cm,
                                           uint32_t cv, bool flip) {
    // each body loads its own matrix, so no matrix is live across the chain
    if (!LEAN && (kbit & (1u << K_DENSE))) {
        Real m[8];
        load_matrix_flip<Real>(mp, m, flip);
        reg_dense<Real, A2, R, T, CTRL>(a, m, cm, cv);
    }
    if (!LEAN && (kbit & (1u << K_REAL))) {
        Real m[8];
        load_matrix_flip<Real>(mp, m, flip);
        reg_real<Real, A2, R, T, CTRL>(a, m, cm, cv);
    }
    if (kbit & (1u << K_DIAG)) {
        Real m[8];
        load_matrix_flip<Real>(mp, m, flip);
        reg_diag<Real, A2, R, T, CTRL>(a, m, cm, cv);
    }
    if (kbit & (1u << K_PHASE)) {
        Real m[8];
        load_matrix<Real>(mp, m);
        reg_phase<Real, A2, R, T, CTRL>(a, m, cm, cv);
    }
    if (!LEAN && (kbit & (1u << K_ANTI))) {
        Real m[8];
        load_matrix_flip<Real>(mp, m, flip);
        reg_anti<Real, A2, R, T, CTRL>(a, m, cm, cv);
    }
    if (kbit & (1u << K_SWAP)) reg_swap<A2, R, T, CTRL>(a, cm, cv);
}

// Target dispatch, the same way: one bit test per register bit.
template <typename Real, typename A2, int R, int T, bool LEAN>
struct RegTarget {
    __device__ __forceinline__ static void run(uint32_t tbit, uint32_t kbit, A2 (&a)[1 << R],
                                               const Real *__restrict__ mp, uint32_t cm, uint32_t cv, bool flip) {
        // one instantiation, with the per-pair control test: gates without
        // register controls (cm = 0, every pair passes) are rare here, since
        // uncontrolled dense gates go out as layers and uncontrolled X gates
        // relabel, and a second copy of every body cost instruction-cache
        // misses
        if (tbit & (1u << T)) reg_kind_c<Real, A2, R, T, true, LEAN>(kbit, a, mp, cm, cv, flip);
        RegTarget<Real, A2, R, T + 1, LEAN>::run(tbit, kbit, a, mp, cm, cv, flip);
    }
};
template <typename Real, typename A2, int R, bool LEAN>
struct RegTarget<Real, A2, R, R, LEAN> {
    __device__ __forceinline__ static void run(uint32_t, uint32_t, A2 (&)[1 << R], const Real *__restrict__,
                                               uint32_t, uint32_t, bool) {}
};

template <typename Real>
__device__ __forceinline__ void load_matrix(const Real *__restrict__ src, Real (&m)[8]);
template <>
__device__ __forceinline__ void load_matrix<double>(const double *__restrict__ src, double (&m)[8]) {
    const double2 *p = reinterpret_cast<const double2 *>(src);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const double2 v = __ldg(p + k);
        m[2 * k] = v.x;
        m[2 * k + 1] = v.y;
    }
}
template <>
__device__ __forceinline__ void load_matrix<float>(const float *__restrict__ src, float (&m)[8]) {
    const float4 *p = reinterpret_cast<const float4 *>(src);
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const float4 v = __ldg(p + k);
        m[4 * k] = v.x;
        m[4 * k + 1] = v.y;
        m[4 * k + 2] = v.z;
        m[4 * k + 3] = v.w;
    }
}

// Loads a gate matrix; with `flip` set, the matrix with both bit values of
// its target exchanged (X M X: m00 <-> m11, m01 <-> m10), for registers whose
// labels have that bit swapped (register relabeling, below).
template <typename Real>
__device__ __forceinline__ void load_matrix_flip(const Real *__restrict__ src, Real (&m)[8], bool flip) {
    // entry k of the swapped matrix is entry 3 - k = k ^ 3 of the stored one
    const int fx = flip ? 3 : 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const typename V2<Real>::T v = load_c<Real, typename V2<Real>::T>(src + 2 * (k ^ fx));
        m[2 * k] = v.x;
        m[2 * k + 1] = v.y;
    }
}

// A layer: uncontrolled dense gates on a set of register bits (mask),
// applied bit 0 first, one straight-line block per active bit (a uniform
// branch skips inactive bits).  Its matrices follow in popcount(mask) records.
template <typename Real, typename A2, int R, int T, bool REAL>
struct LayerStep {
    __device__ __forceinline__ static void run(A2 (&a)[1 << R], const DevOp<Real> *__restrict__ mats, uint32_t mask,
                                               uint32_t xr) {
        if (mask & (1u << T)) {
            Real m[8];
            load_matrix_flip<Real>(mats->m, m, (xr >> T) & 1u);
            if (REAL) reg_real<Real, A2, R, T, false>(a, m, 0u, 0u);
            else reg_dense<Real, A2, R, T, false>(a, m, 0u, 0u);
            mats++;
        }
        LayerStep<Real, A2, R, T + 1, REAL>::run(a, mats, mask, xr);
    }
};
template <typename Real, typename A2, int R, bool REAL>
struct LayerStep<Real, A2, R, R, REAL> {
    __device__ __forceinline__ static void run(A2 (&)[1 << R], const DevOp<Real> *__restrict__, uint32_t,
                                               uint32_t) {}
};

// A layer gate's matrix as loaded: the four complex entries (dense) or their
// real parts (REAL); `get` writes the m[8] form, bit-swapped with `flip`.
template <typename Real, bool REAL>
struct LayerRec;
template <>
struct LayerRec<float, false> {
    float4 a, b;
    __device__ __forceinline__ void load(const DevOp<float> *__restrict__ d) {
        a = __ldg(reinterpret_cast<const float4 *>(d->m));
        b = __ldg(reinterpret_cast<const float4 *>(d->m) + 1);
    }
    __device__ __forceinline__ void get(bool f, float (&m)[8]) const {
        m[0] = f ? b.z : a.x; m[1] = f ? b.w : a.y; m[2] = f ? b.x : a.z; m[3] = f ? b.y : a.w;
        m[4] = f ? a.z : b.x; m[5] = f ? a.w : b.y; m[6] = f ? a.x : b.z; m[7] = f ? a.y : b.w;
    }
};
template <>
struct LayerRec<float, true> {
    float r0, r1, r2, r3;
    __device__ __forceinline__ void load(const DevOp<float> *__restrict__ d) {
        const float4 a = __ldg(reinterpret_cast<const float4 *>(d->m));
        const float4 b = __ldg(reinterpret_cast<const float4 *>(d->m) + 1);
        r0 = a.x; r1 = a.z; r2 = b.x; r3 = b.z;
    }
    __device__ __forceinline__ void get(bool f, float (&m)[8]) const {
        m[0] = f ? r3 : r0; m[2] = f ? r2 : r1; m[4] = f ? r1 : r2; m[6] = f ? r0 : r3;
        m[1] = m[3] = m[5] = m[7] = 0.0f;
    }
};
template <>
struct LayerRec<double, false> {
    double2 e0, e1, e2, e3;
    __device__ __forceinline__ void load(const DevOp<double> *__restrict__ d) {
        const double2 *p = reinterpret_cast<const double2 *>(d->m);
        e0 = __ldg(p); e1 = __ldg(p + 1); e2 = __ldg(p + 2); e3 = __ldg(p + 3);
    }
    __device__ __forceinline__ void get(bool f, double (&m)[8]) const {
        m[0] = f ? e3.x : e0.x; m[1] = f ? e3.y : e0.y; m[2] = f ? e2.x : e1.x; m[3] = f ? e2.y : e1.y;
        m[4] = f ? e1.x : e2.x; m[5] = f ? e1.y : e2.y; m[6] = f ? e0.x : e3.x; m[7] = f ? e0.y : e3.y;
    }
};
template <>
struct LayerRec<double, true> {
    double r0, r1, r2, r3;
    __device__ __forceinline__ void load(const DevOp<double> *__restrict__ d) {
        r0 = __ldg(d->m); r1 = __ldg(d->m + 2); r2 = __ldg(d->m + 4); r3 = __ldg(d->m + 6);
    }
    __device__ __forceinline__ void get(bool f, double (&m)[8]) const {
        m[0] = f ? r3 : r0; m[2] = f ? r2 : r1; m[4] = f ? r1 : r2; m[6] = f ? r0 : r3;
        m[1] = m[3] = m[5] = m[7] = 0.0;
    }
};

template <typename Real, typename A2, int R, int T, bool REAL>
struct LayerStepPre {
    __device__ __forceinline__ static void run(A2 (&a)[1 << R], const DevOp<Real> *__restrict__ mats, uint32_t mask,
                                               uint32_t xr, LayerRec<Real, REAL> &cur) {
        if (mask & (1u << T)) {
            Real m[8];
            cur.get((xr >> T) & 1u, m);
            if (mask >> (T + 1)) cur.load(mats + 1);
            if (REAL) reg_real<Real, A2, R, T, false>(a, m, 0u, 0u);
            else reg_dense<Real, A2, R, T, false>(a, m, 0u, 0u);
            mats++;
        }
        LayerStepPre<Real, A2, R, T + 1, REAL>::run(a, mats, mask, xr, cur);
    }
};
template <typename Real, typename A2, int R, bool REAL>
struct LayerStepPre<Real, A2, R, R, REAL> {
    __device__ __forceinline__ static void run(A2 (&)[1 << R], const DevOp<Real> *__restrict__, uint32_t, uint32_t,
                                               LayerRec<Real, REAL> &) {}
};
// A layer; each active bit's matrix is loaded while the previous bit's
// arithmetic runs, except in FP64 complex layers, where the 16 registers it
// holds cost more in spills than the overlap saves (26-qubit FP64 layered 5%
// slower; FP64 H layers and Grover 5-10% faster, FP32 QFT 2.5% and Grover 9%).
template <typename Real, typename A2, int R, bool REAL>
__device__ __forceinline__ void apply_layer(A2 (&a)[1 << R], const DevOp<Real> *__restrict__ mats, uint32_t mask,
                                            uint32_t xr) {
    if constexpr (sizeof(Real) == 8 && !REAL) {
        LayerStep<Real, A2, R, 0, false>::run(a, mats, mask, xr);
        return;
    }
    LayerRec<Real, REAL> cur;
    cur.load(mats);
    LayerStepPre<Real, A2, R, 0, REAL>::run(a, mats, mask, xr, cur);
}

template <typename Real, typename A2>
__device__ __forceinline__ A2 cmul2(A2 a, A2 b);

// Multiplies the registers whose bit T is 1 by f (a phase diag(1, f)).
template <typename Real, typename A2, int R, int T>
__device__ __forceinline__ void reg_half_phase(A2 (&a)[1 << R], A2 f) {
    const Real nfi = -f.y;
#pragma unroll
    for (int r = 0; r < (1 << R); r++)
        if (r & (1 << T)) ip_cmul(a[r].x, a[r].y, f.x, f.y, nfi);
}

// A split layer (K_LAYER_SPLIT): on each active register bit T the gate
// Rm diag(1, p), Rm real, as a phase on the registers whose bit T is 1 and the
// real gate (2 packed FP32 instructions per amplitude): 4 instructions per
// amplitude against the complex matrix's 8.  (A phase after the real part,
// diag(1, q), follows the layer as a phase record: its code inside every
// bit's body, never run by Rz.Ry gates, made layered passes 7% slower.)
// Seen through a swapped label (xr bit T set) the gate is
//   X Rm diag(1, p) X = p (X Rm X) diag(1, p*),
// so the phase stays on the same registers, conjugated, the real matrix is
// read bit-swapped and p joins the thread's factor `pend`, which the layer
// multiplies into all registers at its end.  Each active bit's record is
// loaded while the previous bit's arithmetic runs (22-26 qubit FP32 layered
// circuits: 7% faster than loading it where it is used).
// one split-gate record: (m00, m01, m10, m11) and p
template <typename Real>
struct SplitRec;
template <>
struct SplitRec<float> {
    float4 r, pq;
    __device__ __forceinline__ void load(const DevOp<float> *__restrict__ d) {
        r = __ldg(reinterpret_cast<const float4 *>(d->m));
        pq = __ldg(reinterpret_cast<const float4 *>(d->m) + 1);
    }
    __device__ __forceinline__ float2 p() const { return make_float2(pq.x, pq.y); }
};
template <>
struct SplitRec<double> {
    double2 r01, r23, pp;
    __device__ __forceinline__ void load(const DevOp<double> *__restrict__ d) {
        const double2 *m = reinterpret_cast<const double2 *>(d->m);
        r01 = __ldg(m);
        r23 = __ldg(m + 1);
        pp = __ldg(m + 2);
    }
    __device__ __forceinline__ double2 p() const { return pp; }
};
template <typename Real>
__device__ __forceinline__ void split_real(const SplitRec<Real> &c, bool flip, Real (&mm)[8]);
template <>
__device__ __forceinline__ void split_real<float>(const SplitRec<float> &c, bool flip, float (&mm)[8]) {
    mm[0] = flip ? c.r.w : c.r.x;
    mm[2] = flip ? c.r.z : c.r.y;
    mm[4] = flip ? c.r.y : c.r.z;
    mm[6] = flip ? c.r.x : c.r.w;
}
template <>
__device__ __forceinline__ void split_real<double>(const SplitRec<double> &c, bool flip, double (&mm)[8]) {
    mm[0] = flip ? c.r23.y : c.r01.x;
    mm[2] = flip ? c.r23.x : c.r01.y;
    mm[4] = flip ? c.r01.y : c.r23.x;
    mm[6] = flip ? c.r01.x : c.r23.y;
}

template <typename Real, typename A2, int R, int T>
struct SplitStep {
    __device__ __forceinline__ static void run(A2 (&a)[1 << R], const DevOp<Real> *__restrict__ mats,
                                               uint32_t mask, uint32_t phases, uint32_t xr, A2 &pend,
                                               SplitRec<Real> &cur) {
        if (mask & (1u << T)) {
            const bool flip = (xr >> T) & 1u;
            const SplitRec<Real> c = cur;
            // the next active bit's record, while this one's arithmetic runs
            if (mask >> (T + 1)) cur.load(mats + 1);
            if (phases & (1u << T)) {
                A2 p = c.p();
                const A2 pf = cmul2<Real>(pend, p);
                pend.x = flip ? pf.x : pend.x;
                pend.y = flip ? pf.y : pend.y;
                p.y = flip ? -p.y : p.y;
                reg_half_phase<Real, A2, R, T>(a, p);
            }
            {
                Real mm[8];
                split_real<Real>(c, flip, mm);
                reg_real<Real, A2, R, T, false>(a, mm, 0u, 0u);
            }
            mats++;
        }
        SplitStep<Real, A2, R, T + 1>::run(a, mats, mask, phases, xr, pend, cur);
    }
};
template <typename Real, typename A2, int R>
struct SplitStep<Real, A2, R, R> {
    __device__ __forceinline__ static void run(A2 (&)[1 << R], const DevOp<Real> *__restrict__, uint32_t, uint32_t,
                                               uint32_t, A2 &, SplitRec<Real> &) {}
};

template <typename Real, typename A2, int R>
__device__ __forceinline__ void apply_split_layer(A2 (&a)[1 << R], const DevOp<Real> *__restrict__ mats,
                                                  uint32_t mask, uint32_t phases, uint32_t xr) {
    A2 pend;
    pend.x = 1;
    pend.y = 0;
    SplitRec<Real> cur;
    cur.load(mats);
    SplitStep<Real, A2, R, 0>::run(a, mats, mask, phases, xr, pend, cur);
    // every thread of the warp reaches this point (ops are uniform)
    if (__any_sync(0xffffffffu, pend.x != (Real)1 || pend.y != (Real)0)) {
#pragma unroll
        for (int r = 0; r < (1 << R); r++) ip_cmul2(a[r], pend);
    }
}

// Phase block: diagonal gates with at most one control, combined per thread
// into a scalar f, per-register-bit factors g[b] (bit 1) and h[b] (bit 0) and
// an optional host-built 2^R table (gates whose target and control are both
// register bits); each register is then multiplied once per involved bit.
// A term applies when its controls on non-tile and thread bits hold; a term
// whose target is not a register bit contributes d1 or d0 according to this
// thread's value of that bit.
template <typename Real, typename A2>
__device__ __forceinline__ A2 load_c(const Real *__restrict__ p);
template <>
__device__ __forceinline__ double2 load_c<double, double2>(const double *__restrict__ p) {
    return __ldg(reinterpret_cast<const double2 *>(p));
}
template <>
__device__ __forceinline__ float2 load_c<float, float2>(const float *__restrict__ p) {
    return __ldg(reinterpret_cast<const float2 *>(p));
}

// Factor of one phase-block term for this thread: d0 or d1 of its diagonal
// gate by the value of its target (a thread or non-tile bit), or 1 when its
// controls on thread and non-tile bits do not hold.  Branch-free: the
// conditions differ between threads of a warp.
template <typename Real, typename A2>
__device__ __forceinline__ A2 term_factor(const DevOp<Real> *__restrict__ t, uint64_t base, uint32_t thr) {
    const uint4 th = __ldg(reinterpret_cast<const uint4 *>(t) + 1);  // cm_thr, cv_thr, tpos2
    const ulonglong2 gl = __ldg(reinterpret_cast<const ulonglong2 *>(t) + 2);
    const A2 f0 = load_c<Real, A2>(t->m), f1 = load_c<Real, A2>(t->m + 6);
    const bool ok = ((base & gl.x) == gl.y) && ((thr & th.x) == th.y);
    const int tp = (int)th.z;
    const uint32_t bv = tp >= TPOS_GLOBAL   ? (uint32_t)(base >> (tp - TPOS_GLOBAL)) & 1u
                        : tp >= TPOS_THREAD ? (thr >> (tp - TPOS_THREAD)) & 1u
                                            : 0u;
    A2 f = bv ? f1 : f0;
    f.x = ok ? f.x : (Real)1;
    f.y = ok ? f.y : (Real)0;
    return f;
}

template <typename Real, typename A2>
__device__ __forceinline__ A2 cmul2(A2 a, A2 b) {
    A2 o;
    o.x = a.x * b.x - a.y * b.y;
    o.y = a.x * b.y + a.y * b.x;
    return o;
}

// acc times the factors of terms t[0..n), two terms per step (two chains, so
// that one term's loads overlap the other's arithmetic).
template <typename Real, typename A2>
__device__ __forceinline__ A2 term_product(const DevOp<Real> *__restrict__ t, int n, uint64_t base, uint32_t thr,
                                           A2 acc) {
    A2 acc2;
    acc2.x = 1;
    acc2.y = 0;
    int i = 0;
#pragma unroll 1
    for (; i + 1 < n; i += 2) {
        const A2 fa = term_factor<Real, A2>(t + i, base, thr), fb = term_factor<Real, A2>(t + i + 1, base, thr);
        acc = cmul2<Real>(acc, fa);
        acc2 = cmul2<Real>(acc2, fb);
    }
    if (i < n) acc = cmul2<Real>(acc, term_factor<Real, A2>(t + i, base, thr));
    return cmul2<Real>(acc, acc2);
}

// D terms (a diagonal gate on register bit b, controls elsewhere): h takes
// d0, g takes d1, where the controls hold.
template <typename Real, typename A2>
__device__ __forceinline__ void term_diag_product(const DevOp<Real> *__restrict__ t, int n, uint64_t base,
                                                  uint32_t thr, A2 &h, A2 &g) {
#pragma unroll 1
    for (int i = 0; i < n; i++) {
        const uint4 th = __ldg(reinterpret_cast<const uint4 *>(t + i) + 1);
        const ulonglong2 gl = __ldg(reinterpret_cast<const ulonglong2 *>(t + i) + 2);
        A2 f0 = load_c<Real, A2>(t[i].m), f1 = load_c<Real, A2>(t[i].m + 6);
        const bool ok = ((base & gl.x) == gl.y) && ((thr & th.x) == th.y);
        f0.x = ok ? f0.x : (Real)1;
        f0.y = ok ? f0.y : (Real)0;
        f1.x = ok ? f1.x : (Real)1;
        f1.y = ok ? f1.y : (Real)0;
        h = cmul2<Real>(h, f0);
        g = cmul2<Real>(g, f1);
    }
}

// A phase block's 2^R table: complex factors by register label, four per
// record (the m[] of consecutive records from z), register r holding label
// r ^ xr.  When no lane of the warp has a relabeled register (xr == 0, as in
// the QFT's phase passes), the labels are the register numbers and every
// entry sits at a constant offset: two entries per 16-byte load in FP32 and
// no address arithmetic, which was most of the integer work of a QFT pass
// (six instructions per register and table).
template <typename Real, typename A2, int R>
__device__ __forceinline__ void apply_table(A2 (&a)[1 << R], const Real *__restrict__ z, uint32_t xr) {
    constexpr int stride = (int)(sizeof(DevOp<Real>) / sizeof(Real));
    if (__all_sync(0xffffffffu, xr == 0u)) {
        if constexpr (sizeof(Real) == 4) {
#pragma unroll
            for (int r = 0; r < (1 << R); r += 2) {
                const float4 f = __ldg(reinterpret_cast<const float4 *>(z + (r >> 2) * stride + 2 * (r & 3)));
                ip_cmul2(a[r], make_float2(f.x, f.y));
                ip_cmul2(a[r + 1], make_float2(f.z, f.w));
            }
        } else {
#pragma unroll
            for (int r = 0; r < (1 << R); r++) ip_cmul2(a[r], load_c<Real, A2>(z + (r >> 2) * stride + 2 * (r & 3)));
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < (1 << R); r++) {
        const uint32_t l = r ^ xr;
        ip_cmul2(a[r], load_c<Real, A2>(z + (l >> 2) * stride + 2 * (l & 3)));
    }
}

// Byte K of the 16 phase-block term counts, kept packed in four words.
template <int K>
__device__ __forceinline__ int count_byte(const uint4 &c) {
    const uint32_t w = K < 4 ? c.x : K < 8 ? c.y : K < 12 ? c.z : c.w;
    return (int)((w >> (8 * (K & 3))) & 0xffu);
}

// Register bit B of a phase block: when the block marks B active, folds the
// G[B], H[B] and D[B] terms into g (factor of the registers whose bit B is 1)
// and h (bit B is 0), starting from `carry` (the block's F factor, handed to
// the first active bit and reset), and multiplies them into the registers
// with one sweep.  Inactive bits cost nothing but the pointer step.
template <typename Real, typename A2, int R, int B>
struct PhaseBits {
    __device__ __forceinline__ static void run(A2 (&a)[1 << R], const DevOp<Real> *__restrict__ t,
                                               const uint4 &cnt, uint32_t act, A2 &carry, uint64_t base,
                                               uint32_t thr, uint32_t xr) {
        const int ng = count_byte<1 + B>(cnt), nh = count_byte<1 + R + B>(cnt), nd = count_byte<1 + 2 * R + B>(cnt);
        if (act & (1u << B)) {
            A2 g = term_product<Real, A2>(t, ng, base, thr, carry);
            A2 h = term_product<Real, A2>(t + ng, nh, base, thr, carry);
            carry.x = 1;
            carry.y = 0;
            term_diag_product<Real, A2>(t + ng + nh, nd, base, thr, h, g);
            // g belongs to the registers whose label has bit B set
            const bool flip = (xr >> B) & 1u;
            const A2 g1 = flip ? h : g, h1 = flip ? g : h;
#pragma unroll
            for (int r = 0; r < (1 << R); r++) ip_cmul2(a[r], ((r >> B) & 1) ? g1 : h1);
        }
        PhaseBits<Real, A2, R, B + 1>::run(a, t + ng + nh + nd, cnt, act, carry, base, thr, xr);
    }
};
template <typename Real, typename A2, int R>
struct PhaseBits<Real, A2, R, R> {
    __device__ __forceinline__ static void run(A2 (&)[1 << R], const DevOp<Real> *__restrict__, const uint4 &,
                                               uint32_t, A2 &, uint64_t, uint32_t, uint32_t) {}
};

// ---- phase blocks of compact phase terms (head flag PB_ANGLES) ------------
// Each term adds a0 or a1 turns to its category's phase where its control
// holds; the index bits it tests are those of the thread's register-0
// amplitude, ix = tile base | the thread bits placed at their index bits
// (head bytes 16..23).  A category's factor is exp(2 pi i * turns), one
// sincospi per category instead of a complex multiply per term.
// The words of one compact term.  A linear term (cbit == PB_LINEAR) keeps its
// index mask where a0 (and, in FP32, a1) sit and its scale in pad2 (FP32) or
// a1 (FP64).
template <typename Real>
struct TermWords;
template <>
struct TermWords<float> {
    uint32_t head;
    float a0, a1, scale;
    uint64_t mask;
    __device__ __forceinline__ TermWords(const unsigned char *p) {
        const uint4 v = __ldg(reinterpret_cast<const uint4 *>(p));
        head = v.x;
        a0 = __uint_as_float(v.y);
        a1 = __uint_as_float(v.z);
        mask = ((uint64_t)v.z << 32) | v.y;
        scale = __uint_as_float(v.w);
    }
};
template <>
struct TermWords<double> {
    uint32_t head;
    double a0, a1, scale;
    uint64_t mask;
    __device__ __forceinline__ TermWords(const unsigned char *p) {
        const uint4 v = __ldg(reinterpret_cast<const uint4 *>(p));
        const double2 w = __ldg(reinterpret_cast<const double2 *>(p) + 1);
        head = v.x;
        a0 = __hiloint2double((int)v.w, (int)v.z);
        a1 = w.x;
        mask = ((uint64_t)v.w << 32) | v.z;
        scale = w.x;
    }
};

// Turns of a linear term at index ix: scale times the masked index as an
// integer, or bit-reversed (brev64 * 2^-63: index bit b weighs 2^-b).
template <typename Real>
__device__ __forceinline__ Real linear_turns(const TermWords<Real> &t, uint64_t ix, bool rev) {
    const unsigned long long x = ix & t.mask;
    const Real v = rev ? (Real)__brevll(x) * (Real)1.0842021724855044e-19 : (Real)x;
    return t.scale * v;
}

// Term k of the block whose terms start at rec0, for a category that adds
// a0 / a1 turns by the value of the term's target: the turns it adds at ix
// (0 where its control does not hold).
template <typename Real>
__device__ __forceinline__ Real term_turns(const unsigned char *__restrict__ rec0, int k, uint64_t ix) {
    constexpr int per = pb_terms_per_record<Real>();
    const TermWords<Real> t(rec0 + (k / per) * sizeof(DevOp<Real>) + (k % per) * sizeof(PhaseTerm<Real>));
    const int cbit = (int)(int8_t)(t.head & 0xffu), cval = (int)((t.head >> 8) & 0xffu);
    const int tbit = (int)(int8_t)((t.head >> 16) & 0xffu);
    const uint32_t tv = tbit < 0 ? 0u : (uint32_t)((ix >> (tbit & 63)) & 1u);
    if (cbit == PB_LINEAR) return (tbit < 0 || tv) ? linear_turns<Real>(t, ix, cval & 1) : (Real)0;
    const bool c = cbit < 0 || (int)((ix >> (cbit & 63)) & 1u) == cval;
    return c ? (tv ? t.a1 : t.a0) : (Real)0;
}

// Term k of a D category (a diagonal on the category's register bit): adds
// its d0 turns to h and its d1 turns to g where its control holds.
template <typename Real>
__device__ __forceinline__ void dterm_turns(const unsigned char *__restrict__ rec0, int k, uint64_t ix, Real &h,
                                            Real &g) {
    constexpr int per = pb_terms_per_record<Real>();
    const TermWords<Real> t(rec0 + (k / per) * sizeof(DevOp<Real>) + (k % per) * sizeof(PhaseTerm<Real>));
    const int cbit = (int)(int8_t)(t.head & 0xffu), cval = (int)((t.head >> 8) & 0xffu);
    if (cbit == PB_LINEAR) {
        const int tbit = (int)(int8_t)((t.head >> 16) & 0xffu);
        if (tbit < 0 || ((ix >> (tbit & 63)) & 1u)) g += linear_turns<Real>(t, ix, cval & 1);
        return;
    }
    const bool c = cbit < 0 || (int)((ix >> (cbit & 63)) & 1u) == cval;
    h += c ? t.a0 : (Real)0;
    g += c ? t.a1 : (Real)0;
}

template <typename Real>
__device__ __forceinline__ Real turns_sum(const unsigned char *__restrict__ rec0, int k0, int n, uint64_t ix, Real acc) {
    Real acc2 = 0;
    int k = 0;
#pragma unroll 1
    for (; k + 1 < n; k += 2) {
        acc += term_turns<Real>(rec0, k0 + k, ix);
        acc2 += term_turns<Real>(rec0, k0 + k + 1, ix);
    }
    if (k < n) acc += term_turns<Real>(rec0, k0 + k, ix);
    return acc + acc2;
}

template <typename A2, typename Real>
__device__ __forceinline__ A2 cis_turns(Real t) {
    const Real r = t - rint(t);
    A2 f;
    if constexpr (sizeof(Real) == 4) sincospif(2.0f * r, &f.y, &f.x);
    else sincospi(2.0 * r, &f.y, &f.x);
    return f;
}

template <typename Real, typename A2, int R, int B>
struct PhaseBitsAngles {
    __device__ __forceinline__ static void run(A2 (&a)[1 << R], const unsigned char *__restrict__ rec0, int k,
                                               const uint4 &cnt, uint32_t act, Real &carry, uint64_t ix, uint32_t xr) {
        const int ng = count_byte<1 + B>(cnt), nh = count_byte<1 + R + B>(cnt), nd = count_byte<1 + 2 * R + B>(cnt);
        if (act & (1u << B)) {
            Real g = turns_sum<Real>(rec0, k, ng, ix, carry);
            Real h = turns_sum<Real>(rec0, k + ng, nh, ix, carry);
            carry = 0;
#pragma unroll 1
            for (int i = 0; i < nd; i++) dterm_turns<Real>(rec0, k + ng + nh + i, ix, h, g);
            // g belongs to the registers whose label has bit B set
            const bool flip = (xr >> B) & 1u;
            const A2 gf = cis_turns<A2>(g), hf = cis_turns<A2>(h);
            const A2 g1 = flip ? hf : gf, h1 = flip ? gf : hf;
#pragma unroll
            for (int r = 0; r < (1 << R); r++) ip_cmul2(a[r], ((r >> B) & 1) ? g1 : h1);
        }
        PhaseBitsAngles<Real, A2, R, B + 1>::run(a, rec0, k + ng + nh + nd, cnt, act, carry, ix, xr);
    }
};
template <typename Real, typename A2, int R>
struct PhaseBitsAngles<Real, A2, R, R> {
    __device__ __forceinline__ static void run(A2 (&)[1 << R], const unsigned char *__restrict__, int, const uint4 &,
                                               uint32_t, Real &, uint64_t, uint32_t) {}
};

// Byte k (runtime) of the 16 phase-block term counts.
__device__ __forceinline__ int count_byte_at(const uint4 &c, int k) {
    const uint32_t w = k < 4 ? c.x : k < 8 ? c.y : k < 12 ? c.z : c.w;
    return (int)((w >> (8 * (k & 3))) & 0xffu);
}

// A gated block's sweep (PB_GATED, no relabeled register in the warp): the
// registers whose bit B is 1 times c and their table entry (read at constant
// offsets).  A gated block always has a table (of ones if nothing else): one
// body instead of a second one without the table, whose code alone slowed
// the QFT's passes.
template <typename Real, typename A2, int R, int B>
struct GatedSweep {
    __device__ __forceinline__ static void run(int b, A2 (&a)[1 << R], A2 c, const Real *__restrict__ z) {
        if (b == B) {
            constexpr int stride = (int)(sizeof(DevOp<Real>) / sizeof(Real));
#pragma unroll
            for (int r = 0; r < (1 << R); r++)
                if (r & (1 << B)) {
                    ip_cmul2(a[r], load_c<Real, A2>(z + (r >> 2) * stride + 2 * (r & 3)));
                    ip_cmul2(a[r], c);
                }
            return;
        }
        GatedSweep<Real, A2, R, B + 1>::run(b, a, c, z);
    }
};
template <typename Real, typename A2, int R>
struct GatedSweep<Real, A2, R, R> {
    __device__ __forceinline__ static void run(int, A2 (&)[1 << R], A2, const Real *__restrict__) {}
};

template <typename Real, typename A2, int R>
__device__ __forceinline__ void apply_phase_block_angles(A2 (&a)[1 << R], const DevOp<Real> *__restrict__ op,
                                                         uint64_t base, uint32_t thr, uint32_t xr) {
    const uint4 hdr = __ldg(reinterpret_cast<const uint4 *>(op));
    const int nrec = (int)hdr.y;
    const bool has_table = hdr.z & PB_HAS_TABLE;
    const uint32_t act = hdr.w;
    const uint4 cnt = __ldg(reinterpret_cast<const uint4 *>(op->m));
    const uint2 tg = __ldg(reinterpret_cast<const uint2 *>(reinterpret_cast<const unsigned char *>(op->m) + 16));
    uint64_t ix = base;
#pragma unroll
    for (int t = 0; t < 8; t++) {
        const uint32_t g = ((t < 4 ? tg.x : tg.y) >> (8 * (t & 3))) & 63u;
        ix |= (uint64_t)((thr >> t) & 1u) << g;
    }
    const unsigned char *rec0 = reinterpret_cast<const unsigned char *>(op + 1);
    if ((hdr.z & PB_GATED) && __all_sync(0xffffffffu, xr == 0u)) {
        // only G[b] terms, then D[b] terms (the walk order with every other
        // category empty); one factor for the registers whose bit b is 1
        const int b = (int)((hdr.z >> PB_GATE_SHIFT) & 7u);
        const int ng = count_byte_at(cnt, 1 + b), nd = count_byte_at(cnt, 1 + 2 * R + b);
        Real g = turns_sum<Real>(rec0, 0, ng, ix, (Real)0), h = 0;
#pragma unroll 1
        for (int i = 0; i < nd; i++) dterm_turns<Real>(rec0, ng + i, ix, h, g);
        GatedSweep<Real, A2, R, 0>::run(b, a, cis_turns<A2>(g), (op + 1 + nrec - (1 << R) / 4)->m);
        return;
    }
    const int nf = count_byte<0>(cnt);
    Real carry = turns_sum<Real>(rec0, 0, nf, ix, (Real)0);
    PhaseBitsAngles<Real, A2, R, 0>::run(a, rec0, nf, cnt, act, carry, ix, xr);
    if ((act & PB_F_ACTIVE) && !(act & ((1u << R) - 1u))) {
        const A2 f = cis_turns<A2>(carry);
#pragma unroll
        for (int r = 0; r < (1 << R); r++) ip_cmul2(a[r], f);
    }
    if (has_table) apply_table<Real, A2, R>(a, (op + 1 + nrec - (1 << R) / 4)->m, xr);
}

// K_PHASE_BLOCK: the F terms fold into one per-thread factor; each active
// register bit costs one sweep of the registers (PhaseBits); the F factor
// rides on the first active bit's sweep, or gets a sweep of its own when no
// bit is active; the thread-independent 2^R table, if any, is one more sweep.
template <typename Real, typename A2, int R>
__device__ __forceinline__ int apply_phase_block(A2 (&a)[1 << R], const DevOp<Real> *__restrict__ op, uint64_t base,
                                                 uint32_t thr, uint32_t xr) {
    const uint4 hdr = __ldg(reinterpret_cast<const uint4 *>(op));
    const int nrec = (int)hdr.y;  // records after the head
    const bool has_table = hdr.z & 1u;
    const uint32_t act = hdr.w;   // active register bits, PB_F_ACTIVE: F terms
    const uint4 cnt = __ldg(reinterpret_cast<const uint4 *>(op->m));  // 16 count bytes
    const DevOp<Real> *__restrict__ t = op + 1;
    A2 carry;
    carry.x = 1;
    carry.y = 0;
    const int nf = count_byte<0>(cnt);
    carry = term_product<Real, A2>(t, nf, base, thr, carry);
    PhaseBits<Real, A2, R, 0>::run(a, t + nf, cnt, act, carry, base, thr, xr);
    if ((act & PB_F_ACTIVE) && !(act & ((1u << R) - 1u))) {
#pragma unroll
        for (int r = 0; r < (1 << R); r++) ip_cmul2(a[r], carry);
    }
    if (has_table) apply_table<Real, A2, R>(a, (t + nrec - (1 << R) / 4)->m, xr);
    return 1 + nrec;
}

// Records taken by the op whose head record is `hdr`: a phase block's terms
// and table, a layer's matrices, or the record alone.
__device__ __forceinline__ int op_records(const uint4 &hdr) {
    if ((int)hdr.x == K_PHASE_BLOCK) return 1 + (int)hdr.y;
    if ((int)hdr.x == K_LAYER || (int)hdr.x == K_LAYER_REAL || (int)hdr.x == K_LAYER_SPLIT) return 1 + __popc(hdr.z);
    return 1;
}

// Applies record `op` (and, for a layer or phase block, the records that
// follow it); its head record `hdr` is already loaded.
//
// Register relabeling: a thread keeps `xr`, and register r holds the
// amplitude whose register label is r ^ xr.  An X on a register bit whose
// controls (if any) lie on thread or non-tile bits -- most CNOTs of a pass --
// only flips a bit of xr.  Gates on a register bit whose xr bit is set use
// the bit-swapped matrix, register-bit control values are read through xr,
// and the next transpose or the store puts every amplitude where its label
// says (xr is then 0 again).
//
// LEAN (Plan::lean): the build for plans whose phase blocks are all compact
// terms, with no controlled dense, real or anti-diagonal gate on a register
// bit and no complex layer.  Leaving those bodies out of the kernel
// -- code the benchmark circuits never run -- made 26-qubit FP32 layered
// passes 5% and QFT passes 9% faster (fewer instruction-fetch stalls), so
// each plan runs the smallest build it can.
template <typename Real, typename A2, int R, bool LEAN>
__device__ __forceinline__ void apply_op(A2 (&a)[1 << R], const DevOp<Real> *__restrict__ op, const uint4 hdr,
                                         uint64_t base, uint32_t thr, uint32_t &xr) {
    const int kind = (int)hdr.x, tpos = (int)hdr.y;  // hdr: kind, tpos, cm_reg, cv_reg of `op`
    if (kind == K_PHASE_BLOCK) {
        if (LEAN || (hdr.z & PB_ANGLES)) apply_phase_block_angles<Real, A2, R>(a, op, base, thr, xr);
        else apply_phase_block<Real, A2, R>(a, op, base, thr, xr);
        return;
    }
    if (kind == K_XSET) {
        // up to 8 (FP32) or 16 (FP64) relabeling X gates, 4 bytes each
        const uint4 *e = reinterpret_cast<const uint4 *>(op->m);
        const int n = tpos;
#pragma unroll
        for (int q = 0; q < xset_entries<Real>() / 4; q++) {
            if (4 * q >= n) break;
            const uint4 w4 = __ldg(e + q);
            const uint32_t w[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (4 * q + j >= n) break;
                const uint32_t t = w[j] & 0xffu, ck = (w[j] >> 8) & 0xffu, cb = (w[j] >> 16) & 0xffu,
                               cv = w[j] >> 24;
                const uint32_t v = ck == XSET_CTRL_THREAD   ? (thr >> cb) & 1u
                                   : ck == XSET_CTRL_GLOBAL ? (uint32_t)(base >> cb) & 1u
                                                            : cv;
                xr ^= (uint32_t)(v == cv) << t;
            }
        }
        return;
    }
    if (kind == K_LAYER_SPLIT) {
        apply_split_layer<Real, A2, R>(a, op + 1, hdr.z, hdr.w, xr);
        return;
    }
    if (kind == K_LAYER || kind == K_LAYER_REAL) {
        const uint32_t mask = hdr.z;  // active register bits
        if (kind == K_LAYER) {
            if constexpr (!LEAN) apply_layer<Real, A2, R, false>(a, op + 1, mask, xr);
        } else {
            apply_layer<Real, A2, R, true>(a, op + 1, mask, xr);
        }
        return;
    }
    const uint4 th = __ldg(reinterpret_cast<const uint4 *>(op) + 1);                 // cm_thr, cv_thr
    const ulonglong2 gl = __ldg(reinterpret_cast<const ulonglong2 *>(op) + 2);       // cm_glob, cv_glob
    if ((base & gl.x) != gl.y) return;
    if ((thr & th.x) != th.y) return;
    const uint32_t cm = hdr.z, cv = hdr.w ^ (xr & hdr.z);
    if (tpos < R) {
        if (kind == K_SWAP && cm == 0) {
            xr ^= 1u << tpos;
            return;
        }
        // a phase gate seen through a swapped label is diag(d1, 1): run it as
        // a diagonal gate on the bit-swapped matrix
        const bool flip = (xr >> tpos) & 1u;
        const int k = (kind == K_PHASE && flip) ? K_DIAG : kind;
        RegTarget<Real, A2, R, 0, LEAN>::run(1u << tpos, 1u << k, a, op->m, cm, cv, flip);
        return;
    }
    // diagonal gate on a thread bit or a non-tile index bit
    const int bv = tpos >= TPOS_GLOBAL ? (int)((base >> (tpos - TPOS_GLOBAL)) & 1)
                                       : (int)((thr >> (tpos - TPOS_THREAD)) & 1);
    if (kind == K_PHASE && !bv) return;
    const A2 f = load_c<Real, A2>(op->m + (bv ? 6 : 0));
    const Real fr = f.x, fi = f.y;
    reg_scale<Real, A2, R, true>(a, fr, fi, cm, cv);
    return;
}

// ---- layout transposes through shared memory --------------------------------

// Moves the registers from layout `from` to layout `to` (layout tables: the
// byte offset of each register bit's unit step, then each thread's register-0
// offset).  Register r holds label r ^ xr (apply_op): its slot is the
// thread's base plus the steps of the bits of r ^ xr, i.e. the base moved by
// the steps of xr plus the steps of r with those bits negated.
template <typename A2, int R>
__device__ __forceinline__ void transpose(A2 (&a)[1 << R], unsigned char *sm, uint32_t thr,
                                          const uint32_t *__restrict__ from, const uint32_t *__restrict__ to,
                                          bool sync_cta_before, bool cross, uint32_t xr) {
    uint32_t wb = __ldg(from + LAYOUT_HDR + thr), s[R];
#pragma unroll
    for (int q = 0; q < R; q++) s[q] = __ldg(from + q);
    if (sync_cta_before) __syncthreads();
    else __syncwarp();
#pragma unroll
    for (int q = 0; q < R; q++) {
        const bool f = (xr >> q) & 1u;
        wb += f ? s[q] : 0u;
        s[q] = f ? 0u - s[q] : s[q];
    }
#pragma unroll
    for (int r = 0; r < (1 << R); r++) {
        uint32_t o = wb;
#pragma unroll
        for (int q = 0; q < R; q++)
            if (r & (1 << q)) o += s[q];
        *reinterpret_cast<A2 *>(sm + o) = a[r];
    }
    uint32_t rb = __ldg(to + LAYOUT_HDR + thr), u[R];
#pragma unroll
    for (int q = 0; q < R; q++) u[q] = __ldg(to + q);
    if (cross) __syncthreads();
    else __syncwarp();
#pragma unroll
    for (int r = 0; r < (1 << R); r++) {
        uint32_t o = rb;
#pragma unroll
        for (int q = 0; q < R; q++)
            if (r & (1 << q)) o += u[q];
        a[r] = *reinterpret_cast<const A2 *>(sm + o);
    }
}

// Index of tile `t`: deposit the bits of t into the non-tile index bits, one
// run of consecutive non-tile bits at a time (uniform across the CTA).
__device__ __forceinline__ uint64_t tile_base(uint64_t t, const PassArgs &pa) {
    uint64_t base = 0;
#pragma unroll
    for (int i = 0; i < MAX_FREE_RUNS; i++) {
        if (i >= pa.nruns) break;
        const int len = pa.run_len[i];
        base |= (t & ((1ull << len) - 1ull)) << pa.run_pos[i];
        t >>= len;
    }
    return base;
}

template <typename Real, int R, int W>
__device__ __forceinline__ void load_tile(typename V2<Real>::T (&a)[1 << R],
                                          const typename V2<Real>::T *__restrict__ state, const PassArgs &pa,
                                          uint64_t base, uint32_t thr) {
    using A2 = typename V2<Real>::T;
    uint64_t off, rs[R];
    thread_geometry<R, W>(pa.ld_gbit, thr, off, rs);
    LoadF<A2, R> f{a, state + (base | off), rs};
    Unroll<1 << R>::run(f);
}

template <typename Real, int R, int W>
__device__ __forceinline__ void store_tile(const typename V2<Real>::T (&a)[1 << R],
                                           typename V2<Real>::T *__restrict__ state, const PassArgs &pa,
                                           uint64_t base, uint32_t xr) {
    using A2 = typename V2<Real>::T;
    // The thread index is re-read so the store geometry is recomputed here
    // instead of being held in registers through every phase.
    uint32_t thr;
    asm volatile("mov.u32 %0, %%tid.x;" : "=r"(thr));
    uint64_t off, rs[R];
    thread_geometry<R, W>(pa.st_gbit, thr, off, rs);
    uint64_t xo = 0;
#pragma unroll
    for (int q = 0; q < R; q++)
        if ((xr >> q) & 1u) xo |= rs[q];
    StoreF<A2, R> f{a, state, base | off | xo, rs};
    Unroll<1 << R>::run(f);
}

// Applies a pass's phases to a tile already in registers (loaded in the
// pass's load layout) and stores it.  `prev_cross`: the CTA's previous use
// of `sm` may still be read by other warps, so the first transpose must
// synchronise the CTA before writing.
// flags, norm_out, scale_in: the pass's PASS_* flags and renormalisation
// slots (the plain pass kernel passes pa's own; the chained kernel computes
// them per position in the pass sequence).  The scale is read through L2:
// in a chained run it was accumulated by other CTAs of the same launch.
template <typename Real, int R, int W, bool LEAN = false>
__device__ __forceinline__ void finish_tile(typename V2<Real>::T (&a)[1 << R], typename V2<Real>::T *__restrict__ state,
                                            const PassArgs &pa, uint64_t base, typename V2<Real>::T *sm,
                                            bool prev_cross, int32_t flags, double *norm_out,
                                            const double *scale_in) {
    using A2 = typename V2<Real>::T;
    constexpr uint32_t LS = LAYOUT_HDR + (32u << W);  // words per layout table
    const uint32_t thr = threadIdx.x, lane = thr & 31;
    const DevOp<Real> *__restrict__ ops = reinterpret_cast<const DevOp<Real> *>(pa.ops);
    unsigned char *smb = reinterpret_cast<unsigned char *>(sm);
    int cur = pa.load_layout;
    if (flags & PASS_SCALE) {
        const Real s = (Real)rsqrt(__ldcg(scale_in));
#pragma unroll
        for (int r = 0; r < (1 << R); r++) {
            a[r].x *= s;
            a[r].y *= s;
        }
    }
    uint32_t xr = 0;  // register relabeling (apply_op)
    for (int p = pa.phase_begin; p < pa.phase_end; p++) {
        const DevPhase ph = pa.phases[p];
        if (ph.layout != cur) {
            transpose<A2, R>(a, smb, thr, pa.layouts + cur * LS, pa.layouts + ph.layout * LS, prev_cross || ph.xwarp,
                             ph.xwarp != 0, xr);
            xr = 0;
            prev_cross = ph.xwarp != 0;
            cur = ph.layout;
        }
        // (loading the next op's head record while this op runs costs more
        // in registers than it saves in load latency)
        for (int i = ph.op_begin; i < ph.op_end;) {
            const uint4 hdr = __ldg(reinterpret_cast<const uint4 *>(ops + i));
            apply_op<Real, A2, R, LEAN>(a, ops + i, hdr, base, thr, xr);
            i += op_records(hdr);
        }
    }
    if (cur != pa.store_layout) {
        transpose<A2, R>(a, smb, thr, pa.layouts + cur * LS, pa.layouts + pa.store_layout * LS,
                         prev_cross || pa.store_xwarp, pa.store_xwarp != 0, xr);
        xr = 0;
    }
    store_tile<Real, R, W>(a, state, pa, base, xr);
    if (flags & PASS_NORM) {
        double acc = 0.0;
#pragma unroll
        for (int r = 0; r < (1 << R); r++) acc += (double)a[r].x * a[r].x + (double)a[r].y * a[r].y;
#pragma unroll
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) atomicAdd(norm_out, acc);
    }
}

// Runs one pass over tile `tile`.  Shared by the plain pass kernel and the
// batched persistent kernel.
template <typename Real, int R, int W, bool LEAN = false>
__device__ __forceinline__ void run_tile(typename V2<Real>::T *__restrict__ state, const PassArgs &pa, uint64_t tile,
                                         typename V2<Real>::T *sm, int32_t flags, double *norm_out,
                                         const double *scale_in) {
    using A2 = typename V2<Real>::T;
    const uint64_t base = tile_base(tile, pa);
    A2 a[1 << R];
    load_tile<Real, R, W>(a, state, pa, base, threadIdx.x);
    finish_tile<Real, R, W, LEAN>(a, state, pa, base, sm, false, flags, norm_out, scale_in);
}
template <typename Real, int R, int W, bool LEAN = false>
__device__ __forceinline__ void run_tile(typename V2<Real>::T *__restrict__ state, const PassArgs &pa, uint64_t tile,
                                         typename V2<Real>::T *sm) {
    run_tile<Real, R, W, LEAN>(state, pa, tile, sm, pa.flags, pa.norm_out, pa.scale_in);
}

}  // namespace hgm
