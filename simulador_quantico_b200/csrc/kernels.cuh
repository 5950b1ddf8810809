// Device code of the state-vector engine (sm_100a).
//
// Pass kernel ("warp-tile" design)
// ---------------------------------
// One CTA owns a tile of 2^K amplitudes, K = 10 + W (W = warp bits, CTA of
// 32*2^W threads).  The tile is the set of state indices that agree on every
// index bit outside the pass's K tile bits; local tile bit q is index bit
// tb[q].  Each thread keeps 32 amplitudes in registers.  Which local bits
// are lane, register and warp bits of a thread is one of three layouts:
//
//   C: lanes = local 0..4, regs = local 5..9,      warps = local 10..9+W
//   B: regs  = local 0..4, lanes = local 5..9,     warps = local 10..9+W
//   A: lanes = local 0..4, warps = local 5..4+W,   regs  = local 5+W..9+W
//
// A gate whose target is a register bit is applied entirely in registers.
// Switching layout is a transpose through shared memory: C<->B stays inside
// each warp (__syncwarp), anything with A crosses warps (__syncthreads).
// Layouts C and A have the lanes on local bits 0..4, whose low `low_bits`
// bits are the lowest index bits of the state: global loads and stores are
// issued in those layouts and each warp instruction moves whole 128-byte
// runs.  Shared memory is XOR-swizzled, phys(j) = j ^ ((j >> 5) & S) with
// S = 7 (16-byte FP64 amplitudes) or 15 (8-byte FP32 amplitudes), which
// keeps every layout's warp access free of bank conflicts.
//
// The state is read once and written once per pass (the reference's
// "load a tile, apply the whole gate batch, write back once",
// src/core/kernel.cu:68-128), so a pass moves 2*S bytes of HBM traffic.
#pragma once

#include <cuda_runtime.h>

#include "hgm_internal.h"

namespace hgm {

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

template <typename Real>
__device__ __forceinline__ uint32_t swz(uint32_t j) {
    constexpr uint32_t S = sizeof(Real) == 8 ? 7u : 15u;
    return j ^ ((j >> 5) & S);
}

template <int W, int LAY>
__device__ __forceinline__ uint32_t local_index(uint32_t lane, uint32_t warp, uint32_t r) {
    if (LAY == LAYOUT_C) return lane | (r << 5) | (warp << 10);
    if (LAY == LAYOUT_B) return r | (lane << 5) | (warp << 10);
    return lane | (warp << 5) | (r << (5 + W));
}

// Offset (in amplitudes) of a thread's register-0 amplitude and the five
// register-bit strides, for a global-capable layout (C or A).
template <int W>
__device__ __forceinline__ void thread_geometry(const PassArgs &pa, int lay, uint32_t lane, uint32_t warp,
                                                uint64_t &off, uint64_t (&rs)[5]) {
    const int ls = 0, ws = (lay == LAYOUT_A) ? 5 : 10, rsb = (lay == LAYOUT_A) ? 5 + W : 5;
    off = 0;
#pragma unroll
    for (int q = 0; q < 5; q++) off |= (uint64_t)((lane >> q) & 1) << pa.tb[ls + q];
#pragma unroll
    for (int q = 0; q < W; q++) off |= (uint64_t)((warp >> q) & 1) << pa.tb[ws + q];
#pragma unroll
    for (int q = 0; q < 5; q++) rs[q] = (uint64_t)1 << pa.tb[rsb + q];
}

template <int r>
__device__ __forceinline__ uint64_t reg_offset(const uint64_t (&rs)[5]) {
    return ((r & 1) ? rs[0] : 0) + ((r & 2) ? rs[1] : 0) + ((r & 4) ? rs[2] : 0) + ((r & 8) ? rs[3] : 0) +
           ((r & 16) ? rs[4] : 0);
}

template <typename A2, int r>
struct Unroll {
    template <typename F>
    __device__ __forceinline__ static void run(F &f) {
        Unroll<A2, r - 1>::run(f);
        f.template go<r - 1>();
    }
};
template <typename A2>
struct Unroll<A2, 0> {
    template <typename F>
    __device__ __forceinline__ static void run(F &) {}
};

template <typename A2>
struct LoadF {
    A2 (&a)[32];
    const A2 *__restrict__ p;
    const uint64_t (&rs)[5];
    template <int r>
    __device__ __forceinline__ void go() {
        a[r] = p[reg_offset<r>(rs)];
    }
};
template <typename A2>
struct StoreF {
    const A2 (&a)[32];
    A2 *__restrict__ p;
    const uint64_t (&rs)[5];
    template <int r>
    __device__ __forceinline__ void go() {
        p[reg_offset<r>(rs)] = a[r];
    }
};

// ---- gate application on register bits -----------------------------------

template <typename Real, typename A2>
__device__ __forceinline__ A2 cmul(A2 a, Real mr, Real mi) {
    A2 o;
    o.x = a.x * mr - a.y * mi;
    o.y = a.x * mi + a.y * mr;
    return o;
}

template <typename Real, typename A2, int T>
__device__ __forceinline__ void reg_dense(A2 (&a)[32], const Real (&m)[8], uint32_t cm, uint32_t cv) {
#pragma unroll
    for (int r = 0; r < 32; r++) {
        if (r & (1 << T)) continue;
        const int r1 = r | (1 << T);
        if ((r & cm) == cv) {
            const A2 x = a[r], y = a[r1];
            A2 o0, o1;
            o0.x = m[0] * x.x - m[1] * x.y + m[2] * y.x - m[3] * y.y;
            o0.y = m[0] * x.y + m[1] * x.x + m[2] * y.y + m[3] * y.x;
            o1.x = m[4] * x.x - m[5] * x.y + m[6] * y.x - m[7] * y.y;
            o1.y = m[4] * x.y + m[5] * x.x + m[6] * y.y + m[7] * y.x;
            a[r] = o0;
            a[r1] = o1;
        }
    }
}

template <typename Real, typename A2, int T>
__device__ __forceinline__ void reg_real(A2 (&a)[32], const Real (&m)[8], uint32_t cm, uint32_t cv) {
#pragma unroll
    for (int r = 0; r < 32; r++) {
        if (r & (1 << T)) continue;
        const int r1 = r | (1 << T);
        if ((r & cm) == cv) {
            const A2 x = a[r], y = a[r1];
            A2 o0, o1;
            o0.x = m[0] * x.x + m[2] * y.x;
            o0.y = m[0] * x.y + m[2] * y.y;
            o1.x = m[4] * x.x + m[6] * y.x;
            o1.y = m[4] * x.y + m[6] * y.y;
            a[r] = o0;
            a[r1] = o1;
        }
    }
}

template <typename Real, typename A2, int T>
__device__ __forceinline__ void reg_diag(A2 (&a)[32], const Real (&m)[8], uint32_t cm, uint32_t cv) {
#pragma unroll
    for (int r = 0; r < 32; r++) {
        if ((r & cm) == cv) {
            if (r & (1 << T)) a[r] = cmul<Real>(a[r], m[6], m[7]);
            else a[r] = cmul<Real>(a[r], m[0], m[1]);
        }
    }
}

template <typename Real, typename A2, int T>
__device__ __forceinline__ void reg_phase(A2 (&a)[32], const Real (&m)[8], uint32_t cm, uint32_t cv) {
#pragma unroll
    for (int r = 0; r < 32; r++) {
        if (!(r & (1 << T))) continue;
        if ((r & cm) == cv) a[r] = cmul<Real>(a[r], m[6], m[7]);
    }
}

template <typename Real, typename A2, int T>
__device__ __forceinline__ void reg_anti(A2 (&a)[32], const Real (&m)[8], uint32_t cm, uint32_t cv) {
#pragma unroll
    for (int r = 0; r < 32; r++) {
        if (r & (1 << T)) continue;
        const int r1 = r | (1 << T);
        if ((r & cm) == cv) {
            const A2 x = a[r], y = a[r1];
            a[r] = cmul<Real>(y, m[2], m[3]);
            a[r1] = cmul<Real>(x, m[4], m[5]);
        }
    }
}

template <typename A2, int T>
__device__ __forceinline__ void reg_swap(A2 (&a)[32], uint32_t cm, uint32_t cv) {
#pragma unroll
    for (int r = 0; r < 32; r++) {
        if (r & (1 << T)) continue;
        const int r1 = r | (1 << T);
        if ((r & cm) == cv) {
            const A2 x = a[r];
            a[r] = a[r1];
            a[r1] = x;
        }
    }
}

// Diagonal gate whose target bit is not a register bit: the factor is the
// same for all of a thread's registers that satisfy the register controls.
template <typename Real, typename A2>
__device__ __forceinline__ void reg_scale(A2 (&a)[32], Real fr, Real fi, uint32_t cm, uint32_t cv) {
#pragma unroll
    for (int r = 0; r < 32; r++)
        if ((r & cm) == cv) a[r] = cmul<Real>(a[r], fr, fi);
}

template <typename Real, typename A2, int T>
__device__ __forceinline__ void reg_kind(int kind, A2 (&a)[32], const Real (&m)[8], uint32_t cm, uint32_t cv) {
    switch (kind) {
        case K_DENSE: reg_dense<Real, A2, T>(a, m, cm, cv); break;
        case K_REAL: reg_real<Real, A2, T>(a, m, cm, cv); break;
        case K_DIAG: reg_diag<Real, A2, T>(a, m, cm, cv); break;
        case K_PHASE: reg_phase<Real, A2, T>(a, m, cm, cv); break;
        case K_ANTI: reg_anti<Real, A2, T>(a, m, cm, cv); break;
        default: reg_swap<A2, T>(a, cm, cv); break;
    }
}

template <typename Real, typename A2>
__device__ __forceinline__ void apply_op(A2 (&a)[32], const DevOp<Real> *__restrict__ op, uint64_t base,
                                         uint32_t thr) {
    const uint64_t cmg = __ldg(reinterpret_cast<const unsigned long long *>(&op->cm_glob));
    const uint64_t cvg = __ldg(reinterpret_cast<const unsigned long long *>(&op->cv_glob));
    if ((base & cmg) != cvg) return;
    const uint4 hdr = __ldg(reinterpret_cast<const uint4 *>(op));  // kind, tpos, cm_reg, cv_reg
    const uint2 th = __ldg(reinterpret_cast<const uint2 *>(&op->cm_thr));
    if ((thr & th.x) != th.y) return;
    const int kind = (int)hdr.x, tpos = (int)hdr.y;
    const uint32_t cm = hdr.z, cv = hdr.w;
    Real m[8];
#pragma unroll
    for (int k = 0; k < 8; k++) m[k] = __ldg(&op->m[k]);
    switch (tpos) {
        case 0: reg_kind<Real, A2, 0>(kind, a, m, cm, cv); return;
        case 1: reg_kind<Real, A2, 1>(kind, a, m, cm, cv); return;
        case 2: reg_kind<Real, A2, 2>(kind, a, m, cm, cv); return;
        case 3: reg_kind<Real, A2, 3>(kind, a, m, cm, cv); return;
        case 4: reg_kind<Real, A2, 4>(kind, a, m, cm, cv); return;
        default: break;
    }
    // diagonal gate on a thread bit or a non-tile index bit
    const int bv = tpos >= TPOS_GLOBAL ? (int)((base >> (tpos - TPOS_GLOBAL)) & 1)
                                       : (int)((thr >> (tpos - TPOS_THREAD)) & 1);
    if (kind == K_PHASE) {
        if (bv) reg_scale<Real>(a, m[6], m[7], cm, cv);
    } else {
        reg_scale<Real>(a, bv ? m[6] : m[0], bv ? m[7] : m[1], cm, cv);
    }
}

// ---- layout transposes through shared memory --------------------------------

template <typename Real, typename A2, int W, int FROM, int TO>
__device__ __forceinline__ void transpose_t(A2 (&a)[32], A2 *sm, uint32_t lane, uint32_t warp, bool sync_cta_before,
                                            bool cross) {
    if (sync_cta_before) __syncthreads();
    else __syncwarp();
#pragma unroll
    for (int r = 0; r < 32; r++) sm[swz<Real>(local_index<W, FROM>(lane, warp, r))] = a[r];
    if (cross) __syncthreads();
    else __syncwarp();
#pragma unroll
    for (int r = 0; r < 32; r++) a[r] = sm[swz<Real>(local_index<W, TO>(lane, warp, r))];
}

template <typename Real, typename A2, int W>
__device__ __forceinline__ void transpose(int from, int to, A2 (&a)[32], A2 *sm, uint32_t lane, uint32_t warp,
                                          bool sync_cta_before, bool cross) {
    if (from == LAYOUT_C && to == LAYOUT_B) transpose_t<Real, A2, W, LAYOUT_C, LAYOUT_B>(a, sm, lane, warp, sync_cta_before, cross);
    else if (from == LAYOUT_B && to == LAYOUT_C) transpose_t<Real, A2, W, LAYOUT_B, LAYOUT_C>(a, sm, lane, warp, sync_cta_before, cross);
    else if (from == LAYOUT_C && to == LAYOUT_A) transpose_t<Real, A2, W, LAYOUT_C, LAYOUT_A>(a, sm, lane, warp, sync_cta_before, cross);
    else if (from == LAYOUT_A && to == LAYOUT_C) transpose_t<Real, A2, W, LAYOUT_A, LAYOUT_C>(a, sm, lane, warp, sync_cta_before, cross);
    else if (from == LAYOUT_B && to == LAYOUT_A) transpose_t<Real, A2, W, LAYOUT_B, LAYOUT_A>(a, sm, lane, warp, sync_cta_before, cross);
    else transpose_t<Real, A2, W, LAYOUT_A, LAYOUT_B>(a, sm, lane, warp, sync_cta_before, cross);
}

// Index of tile `t`: deposit the bits of t into the non-tile index bits.
__device__ __forceinline__ uint64_t tile_base(uint64_t t, uint64_t tile_mask, int n) {
    uint64_t free_bits = ~tile_mask & ((n >= 64) ? ~0ull : ((1ull << n) - 1));
    uint64_t base = 0;
    while (free_bits) {
        const int g = __ffsll((long long)free_bits) - 1;
        free_bits &= free_bits - 1;
        base |= (t & 1ull) << g;
        t >>= 1;
    }
    return base;
}

// Runs one pass over tile `tile`.  Shared by the plain pass kernel and the
// batched persistent kernel.
template <typename Real, int W>
__device__ __forceinline__ void run_tile(typename V2<Real>::T *__restrict__ state, const PassArgs &pa, uint64_t tile,
                                         typename V2<Real>::T *sm) {
    using A2 = typename V2<Real>::T;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t thr = lane | (warp << 5);
    const uint64_t base = tile_base(tile, pa.tile_mask, pa.n);
    const DevOp<Real> *__restrict__ ops = reinterpret_cast<const DevOp<Real> *>(pa.ops);

    A2 a[32];
    int cur = pa.load_layout;
    uint64_t off, rs[5];
    thread_geometry<W>(pa, cur, lane, warp, off, rs);
    {
        LoadF<A2> f{a, state + (base | off), rs};
        Unroll<A2, 32>::run(f);
    }
    if (pa.flags & PASS_SCALE) {
        const Real s = (Real)rsqrt(*pa.scale_in);
#pragma unroll
        for (int r = 0; r < 32; r++) {
            a[r].x *= s;
            a[r].y *= s;
        }
    }
    bool prev_cross = false;
    for (int p = pa.phase_begin; p < pa.phase_end; p++) {
        const DevPhase ph = pa.phases[p];
        if (ph.layout != cur) {
            transpose<Real, A2, W>(cur, ph.layout, a, sm, lane, warp, prev_cross || ph.xwarp, ph.xwarp != 0);
            prev_cross = ph.xwarp != 0;
            cur = ph.layout;
        }
        for (int i = ph.op_begin; i < ph.op_end; i++) apply_op<Real>(a, ops + i, base, thr);
    }
    if (cur != pa.store_layout) {
        const bool cross = (cur == LAYOUT_A) != (pa.store_layout == LAYOUT_A);
        transpose<Real, A2, W>(cur, pa.store_layout, a, sm, lane, warp, prev_cross || cross, cross);
        cur = pa.store_layout;
    }
    if (cur != pa.load_layout) thread_geometry<W>(pa, cur, lane, warp, off, rs);
    {
        StoreF<A2> f{a, state + (base | off), rs};
        Unroll<A2, 32>::run(f);
    }
    if (pa.flags & PASS_NORM) {
        double acc = 0.0;
#pragma unroll
        for (int r = 0; r < 32; r++) acc += (double)a[r].x * a[r].x + (double)a[r].y * a[r].y;
#pragma unroll
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) atomicAdd(pa.norm_out, acc);
    }
}

}  // namespace hgm
