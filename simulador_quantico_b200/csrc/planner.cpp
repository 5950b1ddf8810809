// Planner: compiled op list -> state passes -> register phases.
//
// The reference groups consecutive PTs whose targets fit one
// 2^gpu_region_bits tile (src/core/kernel.cu:195-235) and launches one
// kernel per group.  This planner keeps that idea -- one HBM round trip
// ("pass") applies a whole batch of gates to a tile held on chip -- but
//   * lets gates that commute move past each other (two gates commute when
//     every index bit they share is acted on diagonally by both: controls
//     always are, a target is iff the matrix is diagonal);
//   * treats diagonal gates as tile-independent (they never pair amplitudes,
//     so any pass can apply them whatever its tile bits are);
//   * picks any set of tile bits (not one contiguous window), always keeping
//     the low `low_bits` index bits so every tile is a set of contiguous
//     128-byte runs;
//   * optionally fuses adjacent gates on the same target and controls into
//     one matrix (product formed in FP64).
// Inside a pass, gates are split into register phases of the register-tile
// kernel (kernels.cuh): each phase holds gates whose targets are register
// bits of its layout, a choice of R of the tile's local bits.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>

#include "hgm_internal.h"

namespace hgm {

namespace {

struct SOp {
    int target;
    uint64_t cmask, cval;
    cplx m[4];
    MatClass mc;
    uint64_t nd() const { return mc == MC_DIAG ? 0 : (uint64_t(1) << target); }
    uint64_t dg() const { return cmask | (mc == MC_DIAG ? (uint64_t(1) << target) : 0); }
    uint64_t sup() const { return cmask | (uint64_t(1) << target); }
};

inline bool conflicts(const SOp &o, uint64_t b_nd, uint64_t b_d) {
    return (o.nd() & (b_nd | b_d)) || (o.dg() & b_nd);
}

void matmul2(const cplx a[4], const cplx b[4], cplx out[4]) {  // out = a * b
    cplx r[4] = {a[0] * b[0] + a[1] * b[2], a[0] * b[1] + a[1] * b[3], a[2] * b[0] + a[3] * b[2],
                 a[2] * b[1] + a[3] * b[3]};
    for (int k = 0; k < 4; k++) out[k] = r[k];
}

bool pure_phase_diag(const SOp &s) {
    return s.mc == MC_DIAG && std::abs(std::abs(s.m[0]) - 1.0) < 1e-12 && std::abs(std::abs(s.m[3]) - 1.0) < 1e-12;
}
bool real_dense(const SOp &s) {
    return s.mc == MC_DENSE && s.m[0].imag() == 0 && s.m[1].imag() == 0 && s.m[2].imag() == 0 &&
           s.m[3].imag() == 0;
}

// Merges each gate into the previous gate on the same target with the same
// controls when nothing touched those qubits in between (one record instead
// of two: the per-record work of the pass kernel outweighs the arithmetic a
// cheaper matrix form would save).  fuse == 2 keeps a pure-phase diagonal
// next to a real dense gate (an Rz before an Ry) apart: the real gate then
// takes 4 floating-point instructions per amplitude (2 as packed FP32 pairs)
// instead of the product's 8, and the phase joins a phase block.  Measured
// on 26-qubit FP32 and 30-qubit FP64 random layered circuits that is slower
// (1.07 against 0.79 ms per FP32 pass; 19.2 against 30.9 FP64 layers/s): the
// phase blocks' per-term work outweighs the arithmetic saved, so fuse == 1
// merges every such pair.
std::vector<SOp> fuse_ops(const std::vector<Op> &ops, int fuse) {
    std::vector<SOp> out;
    out.reserve(ops.size());
    int64_t last_touch[64];
    for (int b = 0; b < 64; b++) last_touch[b] = -1;
    for (const Op &op : ops) {
        SOp s;
        s.target = op.target;
        s.cmask = op.cmask;
        s.cval = op.cval;
        for (int k = 0; k < 4; k++) s.m[k] = op.m[k];
        s.mc = classify(s.m);
        if (fuse) {
            int64_t y = last_touch[op.target];
            const bool keep_apart = y >= 0 && fuse == 2 &&
                                    ((pure_phase_diag(out[y]) && real_dense(s)) || (real_dense(out[y]) && pure_phase_diag(s)));
            if (y >= 0 && !keep_apart && out[y].target == s.target && out[y].cmask == s.cmask &&
                out[y].cval == s.cval) {
                bool adjacent = true;
                uint64_t sup = s.sup();
                while (sup) {
                    int b = __builtin_ctzll(sup);
                    sup &= sup - 1;
                    if (last_touch[b] != y) {
                        adjacent = false;
                        break;
                    }
                }
                if (adjacent) {
                    matmul2(s.m, out[y].m, out[y].m);
                    out[y].mc = classify(out[y].m);
                    continue;
                }
            }
        }
        out.push_back(s);
        uint64_t sup = s.sup();
        while (sup) {
            int b = __builtin_ctzll(sup);
            sup &= sup - 1;
            last_touch[b] = (int64_t)out.size() - 1;
        }
    }
    return out;
}

// Role of each local tile bit in a layout (struct Lay): thread bit t (lanes
// 0..4, warps 5..) or register bit q.
enum RoleKind { ROLE_THREAD = 0, ROLE_REG = 1 };
struct Role {
    int kind, idx;
};
struct Roles {
    Role of[MAX_LAYOUT_ROLES];
    int8_t thr_gbit[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // index bit of each thread bit (set by the caller)
    Roles(const Lay &lay, int R, int W) {
        for (int k = 0; k < MAX_LAYOUT_ROLES; k++) of[k] = {ROLE_THREAD, -1};
        for (int k = 0; k < 5 + W + R; k++)
            of[lay.pos[k]] = k < 5 + W ? Role{ROLE_THREAD, k} : Role{ROLE_REG, k - 5 - W};
    }
};

// Builds layouts.  Every layout keeps a warp's shared-memory accesses free of
// bank conflicts: with slot(j) = j + (j >> R) (kernels.cuh pad_slot), the
// unit slot of local bit q is 1, 2, 4, 8 (mod 8 for 16-byte, mod 16 for
// 8-byte amplitudes) exactly for q = i or q = i + R, i < NB, where NB = 3
// (FP64: a quarter warp per 128-byte wavefront) or 4 (FP32: a half warp).
// So thread bit i < NB sits on local bit i, or on i + R when i is a register
// bit, and no layout takes both i and i + R as register bits.  A layout is
// "coalesced" when thread bits 0..L-1 are local bits 0..L-1, the low index
// bits: only such layouts load and store the state.
struct LayoutMaker {
    int R, W, K, NB, L;
    bool feasible(uint32_t S) const {
        if (__builtin_popcount(S) > R) return false;
        for (int i = 0; i < NB; i++)
            if (((S >> i) & 1) && ((S >> (i + R)) & 1)) return false;
        return true;
    }
    bool coalesced(const Lay &lay) const {
        for (int i = 0; i < L && i < 5; i++)
            if (lay.pos[i] != i) return false;
        return true;
    }
    // Register bits S (R of them, feasible); warp bits where `prev` has them
    // when those local bits are free, so that the transpose stays inside
    // each warp.
    Lay make(uint32_t S, const Lay *prev) const {
        Lay lay;
        for (int k = 0; k < MAX_LAYOUT_ROLES; k++) lay.pos[k] = -1;
        uint32_t used = S;
        int k = 5 + W;
        for (int q = 0; q < K; q++)
            if ((S >> q) & 1) lay.pos[k++] = (int8_t)q;
        for (int i = 0; i < NB; i++) {
            const int q = ((S >> i) & 1) ? i + R : i;
            lay.pos[i] = (int8_t)q;
            used |= 1u << q;
        }
        for (int i = NB; i < L && i < 5; i++)
            if (!((used >> i) & 1)) {
                lay.pos[i] = (int8_t)i;
                used |= 1u << i;
            }
        if (prev)
            for (int w = 0; w < W; w++) {
                const int q = prev->pos[5 + w];
                if (!((used >> q) & 1)) {
                    lay.pos[5 + w] = (int8_t)q;
                    used |= 1u << q;
                }
            }
        int q = 0;
        for (int t = 0; t < 5 + W; t++) {
            if (lay.pos[t] >= 0) continue;
            while ((used >> q) & 1) q++;
            lay.pos[t] = (int8_t)q;
            used |= 1u << q;
        }
        return lay;
    }
    // Adds bits to S until it has R, each only if S stays feasible: bits of
    // `first` at or above L, then any bits at or above L, then `first`'s low
    // bits, then any (low bits last keep the layout coalesced).
    uint32_t fill(uint32_t S, uint32_t first) const {
        for (int pass = 0; pass < 4 && __builtin_popcount(S) < R; pass++) {
            for (int q = 0; q < K && __builtin_popcount(S) < R; q++) {
                const bool want = pass == 0   ? (((first >> q) & 1) && q >= L)
                                  : pass == 1 ? q >= L
                                  : pass == 2 ? ((first >> q) & 1)
                                              : true;
                if (want && !((S >> q) & 1) && feasible(S | (1u << q))) S |= 1u << q;
            }
        }
        return S;
    }
    static uint32_t regs(const Lay &lay, int R, int W) {
        uint32_t S = 0;
        for (int q = 0; q < R; q++) S |= 1u << lay.pos[5 + W + q];
        return S;
    }
    bool same_warps(const Lay &a, const Lay &b) const {
        for (int w = 0; w < W; w++)
            if (a.pos[5 + w] != b.pos[5 + w]) return false;
        return true;
    }
};

template <typename Real>
DevOp<Real> encode(const SOp &o, const Roles &ro, const int loc_of[64], uint64_t tile_mask) {
    DevOp<Real> d;
    memset(&d, 0, sizeof d);
    uint64_t cm = o.cmask;
    while (cm) {
        int g = __builtin_ctzll(cm);
        cm &= cm - 1;
        uint32_t v = (o.cval >> g) & 1;
        if (!((tile_mask >> g) & 1)) {
            d.cm_glob |= uint64_t(1) << g;
            d.cv_glob |= uint64_t(v) << g;
            continue;
        }
        const Role rl = ro.of[loc_of[g]];
        if (rl.kind == ROLE_REG) {
            d.cm_reg |= 1u << rl.idx;
            d.cv_reg |= v << rl.idx;
        } else {
            d.cm_thr |= 1u << rl.idx;
            d.cv_thr |= v << rl.idx;
        }
    }
    const cplx *m = o.m;
    bool all_real = m[0].imag() == 0 && m[1].imag() == 0 && m[2].imag() == 0 && m[3].imag() == 0;
    switch (o.mc) {
        case MC_DENSE: d.kind = all_real ? K_REAL : K_DENSE; break;
        case MC_DIAG: d.kind = (m[0] == 1.0) ? K_PHASE : K_DIAG; break;
        default: d.kind = (m[1] == 1.0 && m[2] == 1.0) ? K_SWAP : K_ANTI; break;
    }
    int g = o.target;
    if (!((tile_mask >> g) & 1)) {
        d.tpos = TPOS_GLOBAL + g;  // diagonal gates only
    } else {
        const Role rl = ro.of[loc_of[g]];
        d.tpos = rl.kind == ROLE_REG ? rl.idx : TPOS_THREAD + rl.idx;
    }
    d.tpos2 = d.tpos;
    for (int k = 0; k < 4; k++) {
        d.m[2 * k] = (Real)m[k].real();
        d.m[2 * k + 1] = (Real)m[k].imag();
    }
    return d;
}

// A phase-block term before encoding: turns a0 / a1 added by the value 0 / 1
// of the target (index bit tbit, or the category's register bit when tbit <
// 0), where index bit cbit has value cval (cbit < 0: always).
struct RawTerm {
    int cbit, cval, tbit;
    double a0, a1;
};

// Writes the linear term (PB_LINEAR) of `bits` -> weight into t if the
// weights are scale * 2^b (or scale * 2^-b: `rev`) for one scale.
template <typename Real>
bool make_linear(const std::map<int, double> &w, int cond_bit, PhaseTerm<Real> &t) {
    if (w.size() < 2) return false;
    for (int rev = 0; rev < 2; rev++) {
        const auto first = *w.begin();
        const double scale = rev ? std::ldexp(first.second, first.first) : std::ldexp(first.second, -first.first);
        bool ok = scale != 0.0;
        uint64_t mask = 0;
        for (const auto &kv : w) {
            const double want = rev ? std::ldexp(scale, -kv.first) : std::ldexp(scale, kv.first);
            ok = ok && std::abs(kv.second - want) <= 1e-12 * std::abs(want);
            mask |= uint64_t(1) << kv.first;
        }
        if (!ok) continue;
        memset(&t, 0, sizeof t);
        t.cbit = PB_LINEAR;
        t.cval = (int8_t)rev;
        t.tbit = (int8_t)cond_bit;
        const Real s = (Real)scale;
        unsigned char *p = reinterpret_cast<unsigned char *>(&t);
        memcpy(p + sizeof(Real), &mask, sizeof mask);                         // a0 (and a1 for FP32)
        memcpy(p + (sizeof(Real) == 4 ? 3 : 2) * sizeof(Real), &s, sizeof s);  // pad2 (FP32) or a1 (FP64)
        return true;
    }
    return false;
}

// The compact terms of one category (kind 0: F; 1: G or H; 2: D).  Terms
// that add a1 turns where one more index bit is 1 (a0 = 0) are grouped --
// D: by nothing (the control bit varies), G/H: by nothing (the target bit
// varies), F: by target (the control bit varies) -- and a group whose
// weights form a geometric run becomes one linear term.
template <typename Real>
std::vector<PhaseTerm<Real>> compact_terms(const std::vector<RawTerm> &raw, int kind) {
    std::vector<PhaseTerm<Real>> out;
    std::map<int, std::map<int, double>> groups;  // condition bit -> (varying bit -> summed turns)
    std::vector<bool> grouped(raw.size(), false);
    for (size_t i = 0; i < raw.size(); i++) {
        const RawTerm &t = raw[i];
        if (std::abs(t.a0) > 1e-15) continue;
        int cond = -1, bit = -1;
        if (kind == 2 && t.cbit >= 0 && t.cval == 1 && t.tbit < 0) bit = t.cbit;
        else if (kind == 1 && t.cbit < 0 && t.tbit >= 0) bit = t.tbit;
        else if (kind == 0 && t.cbit >= 0 && t.cval == 1 && t.tbit >= 0) {
            cond = t.tbit;
            bit = t.cbit;
        }
        if (bit < 0) continue;
        groups[cond][bit] += t.a1;
        grouped[i] = true;
    }
    std::map<int, bool> folded;
    for (const auto &g : groups) {
        PhaseTerm<Real> lt;
        folded[g.first] = make_linear<Real>(g.second, g.first, lt);
        if (folded[g.first]) out.push_back(lt);
    }
    for (size_t i = 0; i < raw.size(); i++) {
        const RawTerm &t = raw[i];
        if (grouped[i]) {
            const int cond = kind == 0 ? t.tbit : -1;
            if (folded[cond]) continue;
        }
        PhaseTerm<Real> p;
        memset(&p, 0, sizeof p);
        p.cbit = (int8_t)t.cbit;
        p.cval = (int8_t)t.cval;
        p.tbit = (int8_t)t.tbit;
        p.a0 = (Real)t.a0;
        p.a1 = (Real)t.a1;
        out.push_back(p);
    }
    return out;
}

// Phase block (K_PHASE_BLOCK): diagonal gates with at most one control that
// can all move to the front of what is left, combined into per-thread
// factors (kernels.cuh apply_phase_block).  Returns false when fewer than
// `min_terms` qualify.
template <typename Real>
bool emit_phase_block(const std::vector<SOp> &ops, std::vector<int> &rest, const Roles &ro, int R,
                      const int loc_of[64], uint64_t tmask, int min_terms, std::vector<DevOp<Real>> &out) {
    // category lists: 0 = F, 1 + b = G[b], 1 + R + b = H[b], 1 + 2R + b = D[b]
    std::vector<std::vector<int>> cat(1 + 3 * R);
    std::vector<cplx> table(size_t(1) << R, cplx(1.0, 0.0));
    bool has_table = false;
    std::vector<int> members;
    uint64_t bn = 0, bd = 0;
    auto loc_role = [&](int g, Role &rl) -> bool {  // false: not a tile bit
        if (!((tmask >> g) & 1)) return false;
        rl = ro.of[loc_of[g]];
        return true;
    };
    for (int idx : rest) {
        const SOp &op = ops[idx];
        bool cand = false;
        if (op.mc == MC_DIAG && __builtin_popcountll(op.cmask) <= 1 && !conflicts(op, bn, bd)) {
            Role tr, cr;
            const bool t_reg = loc_role(op.target, tr) && tr.kind == ROLE_REG;
            int c_bit = op.cmask ? __builtin_ctzll(op.cmask) : -1;
            const bool c_reg = c_bit >= 0 && loc_role(c_bit, cr) && cr.kind == ROLE_REG;
            int k = -1;
            if (t_reg && (c_reg || c_bit < 0)) {
                // only register bits: thread-independent, folded into the table
                const int v = c_bit >= 0 ? (int)((op.cval >> c_bit) & 1) : 0;
                for (size_t r = 0; r < table.size(); r++)
                    if (c_bit < 0 || (int)((r >> cr.idx) & 1) == v)
                        table[r] *= ((r >> tr.idx) & 1) ? op.m[3] : op.m[0];
                has_table = true;
                cand = true;
            } else if (t_reg) {
                k = 1 + 2 * R + tr.idx;  // D[t]
            } else if (c_reg) {
                k = ((op.cval >> c_bit) & 1) ? 1 + cr.idx : 1 + R + cr.idx;  // G[c] / H[c]
            } else {
                k = 0;  // F
            }
            if (k >= 0 && cat[k].size() < (size_t)PB_TERMS) {
                cat[k].push_back(idx);
                cand = true;
            }
            if (cand) members.push_back(idx);
        }
        if (!cand) {
            bn |= op.nd();
            bd |= op.dg();
        }
    }
    if ((int)members.size() < min_terms) return false;
    // compact terms when every term's entries are pure phases
    bool angles = true;
    for (const auto &c : cat)
        for (int idx : c)
            for (int k : {0, 3})
                angles = angles && std::abs(std::abs(ops[idx].m[k]) - 1.0) < 1e-12;
    // the compact terms of each category, runs of geometric weights folded
    // into linear terms
    std::vector<std::vector<PhaseTerm<Real>>> ct(1 + 3 * R);
    if (angles) {
        const double turn = 1.0 / (2.0 * 3.14159265358979323846);
        for (int k = 0; k < 1 + 3 * R; k++) {
            std::vector<RawTerm> raw;
            for (int idx : cat[k]) {
                const SOp &op = ops[idx];
                const int c_bit = op.cmask ? __builtin_ctzll(op.cmask) : -1;
                const bool c_reg = c_bit >= 0 && ((tmask >> c_bit) & 1) && ro.of[loc_of[c_bit]].kind == ROLE_REG;
                const bool t_reg = ((tmask >> op.target) & 1) && ro.of[loc_of[op.target]].kind == ROLE_REG;
                RawTerm t;
                t.cbit = c_reg ? -1 : c_bit;  // G/H: the control is the category's register bit
                t.cval = c_bit >= 0 ? (int)((op.cval >> c_bit) & 1) : 0;
                t.tbit = t_reg ? -1 : op.target;
                t.a0 = std::arg(op.m[0]) * turn;
                t.a1 = std::arg(op.m[3]) * turn;
                raw.push_back(t);
            }
            ct[k] = compact_terms<Real>(raw, k == 0 ? 0 : (k <= 2 * R ? 1 : 2));
        }
    }
    // a gate bit: a register bit b such that every factor is 1 where label
    // bit b is 0 (only G[b] and D[b] terms, D terms adding no d0 turns, and
    // a table of exact ones wherever bit b is 0)
    int gate = -1;
    for (int b = 0; angles && b < R && gate < 0; b++) {
        bool ok = true;
        for (int k = 0; k < 1 + 3 * R && ok; k++) {
            if (ct[k].empty() || k == 1 + b) continue;
            if (k != 1 + 2 * R + b) {
                ok = false;
                continue;
            }
            for (const PhaseTerm<Real> &t : ct[k]) ok = ok && (t.cbit == PB_LINEAR || t.a0 == (Real)0);
        }
        for (size_t r = 0; has_table && ok && r < table.size(); r++)
            if (!((r >> b) & 1)) ok = (Real)table[r].real() == (Real)1 && (Real)table[r].imag() == (Real)0;
        if (ok) gate = b;
    }
    // a gated block always carries its table (ones where no term reaches), so
    // that the kernel's gated sweep has one form
    if (gate >= 0) has_table = true;
    DevOp<Real> head;
    memset(&head, 0, sizeof head);
    head.kind = K_PHASE_BLOCK;
    head.cm_reg = (has_table ? PB_HAS_TABLE : 0u) | (angles ? PB_ANGLES : 0u) |
                  (gate >= 0 ? PB_GATED | ((uint32_t)gate << PB_GATE_SHIFT) : 0u);
    uint8_t counts[16] = {0};
    int nrec = 0;
    for (int k = 0; k < 1 + 3 * R; k++) {
        const size_t nk = angles ? ct[k].size() : cat[k].size();
        counts[k] = (uint8_t)nk;
        nrec += (int)nk;
        if (!nk) continue;
        head.cv_reg |= k == 0 ? PB_F_ACTIVE : 1u << ((k - 1) % R);
    }
    const int table_recs = has_table ? (1 << R) / 4 : 0;
    constexpr int per = pb_terms_per_record<Real>();
    if (angles) nrec = (nrec + per - 1) / per;
    head.tpos = nrec + table_recs;
    memcpy(head.m, counts, 16);
    if (angles) memcpy(reinterpret_cast<unsigned char *>(head.m) + 16, ro.thr_gbit, 8);
    out.push_back(head);
    // terms in the kernel's walk order: F, then per register bit b: G[b], H[b], D[b]
    std::vector<int> order(cat[0]);
    for (int b = 0; b < R; b++)
        for (int k : {1 + b, 1 + R + b, 1 + 2 * R + b}) order.insert(order.end(), cat[k].begin(), cat[k].end());
    if (!angles) {
        for (int idx : order) out.push_back(encode<Real>(ops[idx], ro, loc_of, tmask));
    } else {
        // in the kernel's walk order: F, then per register bit b: G[b], H[b], D[b]
        std::vector<PhaseTerm<Real>> terms(ct[0]);
        for (int b = 0; b < R; b++)
            for (int k : {1 + b, 1 + R + b, 1 + 2 * R + b}) terms.insert(terms.end(), ct[k].begin(), ct[k].end());
        for (int r = 0; r < nrec; r++) {
            DevOp<Real> rec;
            memset(&rec, 0, sizeof rec);
            for (int j = 0; j < per && r * per + j < (int)terms.size(); j++)
                memcpy(reinterpret_cast<unsigned char *>(&rec) + j * sizeof(PhaseTerm<Real>), &terms[r * per + j],
                       sizeof(PhaseTerm<Real>));
            out.push_back(rec);
        }
    }
    for (int q = 0; q < table_recs; q++) {
        DevOp<Real> rec;
        memset(&rec, 0, sizeof rec);
        for (int k = 0; k < 4; k++) {
            rec.m[2 * k] = (Real)table[4 * q + k].real();
            rec.m[2 * k + 1] = (Real)table[4 * q + k].imag();
        }
        out.push_back(rec);
    }
    std::vector<int> keep;
    for (int idx : rest)
        if (std::find(members.begin(), members.end(), idx) == members.end()) keep.push_back(idx);
    rest.swap(keep);
    return true;
}

// X gates that only relabel registers (K_XSET): target a register bit of the
// layout, at most one control, on a thread or non-tile bit.  Takes those that
// can move to the front of what is left, up to one record's worth; returns
// whether it emitted a record (one record and no per-gate control checks
// instead of a record per gate).
template <typename Real>
bool emit_xset(const std::vector<SOp> &ops, std::vector<int> &rest, const Roles &ro, const int loc_of[64],
               uint64_t tmask, std::vector<DevOp<Real>> &out) {
    constexpr int cap = xset_entries<Real>();
    std::vector<int> members;
    uint8_t ent[cap][4];
    uint64_t bn = 0, bd = 0;
    for (int idx : rest) {
        if ((int)members.size() == cap) break;
        const SOp &op = ops[idx];
        bool cand = false;
        const bool is_x = op.mc == MC_ANTI && op.m[1] == 1.0 && op.m[2] == 1.0;
        if (is_x && __builtin_popcountll(op.cmask) <= 1 && !conflicts(op, bn, bd) && ((tmask >> op.target) & 1)) {
            const Role tr = ro.of[loc_of[op.target]];
            if (tr.kind == ROLE_REG) {
                uint8_t *e = ent[members.size()];
                e[0] = (uint8_t)tr.idx;
                e[1] = XSET_CTRL_NONE;
                e[2] = e[3] = 0;
                cand = true;
                if (op.cmask) {
                    const int c = __builtin_ctzll(op.cmask);
                    e[3] = (uint8_t)((op.cval >> c) & 1);
                    if (!((tmask >> c) & 1)) {
                        e[1] = XSET_CTRL_GLOBAL;
                        e[2] = (uint8_t)c;
                    } else if (ro.of[loc_of[c]].kind == ROLE_THREAD) {
                        e[1] = XSET_CTRL_THREAD;
                        e[2] = (uint8_t)ro.of[loc_of[c]].idx;
                    } else {
                        cand = false;  // a register-bit control swaps amplitudes
                    }
                }
                if (cand) members.push_back(idx);
            }
        }
        if (!cand) {
            bn |= op.nd();
            bd |= op.dg();
        }
    }
    if (members.empty()) return false;
    DevOp<Real> d;
    memset(&d, 0, sizeof d);
    d.kind = K_XSET;
    d.tpos = (int32_t)members.size();
    memcpy(d.m, ent, members.size() * 4);
    out.push_back(d);
    std::vector<int> keep;
    for (int idx : rest)
        if (std::find(members.begin(), members.end(), idx) == members.end()) keep.push_back(idx);
    rest.swap(keep);
    return true;
}

// Writes M = s diag(1, q) Rm diag(1, p) with Rm real and |s| = |p| = |q| = 1
// (the Z-Y-Z form every unitary has: Rz Ry Rz up to a global phase), with s,
// p and q in the right half plane (a sign goes into Rm) and p or q exactly 1
// when within 1e-15 of it.  False when an entry is 0 or M has no such form
// within 1e-14 of its largest entry.
bool split_gate(const cplx m[4], double rm[4], cplx &s, cplx &p, cplx &q) {
    double big = 0.0;
    for (int k = 0; k < 4; k++) {
        if (m[k] == 0.0) return false;
        big = std::max(big, std::abs(m[k]));
    }
    auto unit = [](cplx z) { return z / std::abs(z); };
    auto right = [](cplx z) { return (z.real() < 0.0 || (z.real() == 0.0 && z.imag() < 0.0)) ? -z : z; };
    s = unit(m[0]);
    p = right(unit(m[1]) / s);
    q = right(unit(m[2]) / s);
    s = right(s);
    if (std::abs(p - 1.0) <= 1e-15) p = 1.0;
    if (std::abs(q - 1.0) <= 1e-15) q = 1.0;
    // m_jk = s q^j p^k rm_jk
    const cplx f[4] = {s, s * p, s * q, s * q * p};
    for (int k = 0; k < 4; k++) {
        rm[k] = (m[k] * std::conj(f[k])).real();
        if (std::abs(m[k] - f[k] * rm[k]) > 1e-14 * big) return false;
    }
    return true;
}

// Emits a phase's gates as a list schedule.  At each step: a phase block if
// at least three diagonal gates (at most one control each) can move to the
// front; else a layer -- the uncontrolled dense gates on distinct register
// bits of the layout that could all move to the front of what is left
// (cm_reg holds the mask of those bits, their matrices follow, lowest
// register bit first) -- if there are at least two; else a phase block of
// two; else a layer of one; else the relabeling X gates that can move to the
// front (K_XSET); else the first remaining gate on its own record.
// With `split`, a layer of complex gates that all have the split form
// (split_gate) goes out as K_LAYER_SPLIT; their scalars s multiply into
// `global`.
template <typename Real>
void emit_phase(const std::vector<SOp> &ops, std::vector<int> rest, const Roles &ro, int R, const int loc_of[64],
                uint64_t tmask, bool split, cplx &global, std::vector<DevOp<Real>> &out) {
    std::vector<int> keep;
    while (!rest.empty()) {
        if (emit_phase_block<Real>(ops, rest, ro, R, loc_of, tmask, 3, out)) continue;
        int slot[8];
        for (int k = 0; k < 8; k++) slot[k] = -1;
        int found = 0;
        bool all_real = true;
        uint64_t bn = 0, bd = 0;
        for (int idx : rest) {
            const SOp &op = ops[idx];
            bool cand = false;
            if (op.mc == MC_DENSE && op.cmask == 0 && !conflicts(op, bn, bd)) {
                const Role rl = ro.of[loc_of[op.target]];
                if (rl.kind == ROLE_REG && slot[rl.idx] < 0) {
                    slot[rl.idx] = idx;
                    found++;
                    cand = true;
                    for (int k = 0; k < 4; k++) all_real = all_real && op.m[k].imag() == 0;
                }
            }
            if (!cand) {
                bn |= op.nd();
                bd |= op.dg();
            }
            if (found == R) break;
        }
        keep.clear();
        // a lone dense gate goes out as a one-gate layer (the cheaper
        // dispatch) when it is the first remaining gate and no phase block of
        // two is available; otherwise the first gate goes out on its own so
        // that a wider layer can still form behind it
        bool lone = false;
        if (found == 1) {
            if (emit_phase_block<Real>(ops, rest, ro, R, loc_of, tmask, 2, out)) continue;
            for (int k = 0; k < R; k++) lone = lone || slot[k] == rest[0];
        }
        if (found >= 2 || lone) {
            DevOp<Real> head;
            memset(&head, 0, sizeof head);
            head.kind = all_real ? K_LAYER_REAL : K_LAYER;
            head.tpos = found;
            for (int k = 0; k < R; k++)
                if (slot[k] >= 0) head.cm_reg |= 1u << k;
            // the split form of every gate of the layer, if all have one
            double rm[8][4];
            cplx sc[8], pp[8], qq[8];
            bool all_split = split && !all_real;
            for (int k = 0; k < R && all_split; k++)
                if (slot[k] >= 0) all_split = split_gate(ops[slot[k]].m, rm[k], sc[k], pp[k], qq[k]);
            if (all_split) {
                head.kind = K_LAYER_SPLIT;
                for (int k = 0; k < R; k++) {
                    if (slot[k] < 0) continue;
                    if (pp[k] != 1.0) head.cv_reg |= 1u << k;
                }
            }
            out.push_back(head);
            for (int k = 0; k < R; k++) {
                if (slot[k] < 0) continue;
                DevOp<Real> d = encode<Real>(ops[slot[k]], ro, loc_of, tmask);
                if (all_split) {
                    for (int j = 0; j < 4; j++) d.m[j] = (Real)rm[k][j];
                    d.m[4] = (Real)pp[k].real();
                    d.m[5] = (Real)pp[k].imag();
                    d.m[6] = (Real)qq[k].real();
                    d.m[7] = (Real)qq[k].imag();
                    global *= sc[k];
                }
                out.push_back(d);
            }
            // a split gate's phase after its real part, diag(1, q), follows
            // the layer as a phase record on the same register bit: the
            // kernel's split layer carries only the phase before
            for (int k = 0; k < R && all_split; k++) {
                if (slot[k] < 0 || qq[k] == 1.0) continue;
                DevOp<Real> d;
                memset(&d, 0, sizeof d);
                d.kind = K_PHASE;
                d.tpos = d.tpos2 = k;
                d.m[0] = (Real)1;
                d.m[6] = (Real)qq[k].real();
                d.m[7] = (Real)qq[k].imag();
                out.push_back(d);
            }
            for (int idx : rest) {
                bool member = false;
                for (int k = 0; k < R; k++) member = member || slot[k] == idx;
                if (!member) keep.push_back(idx);
            }
        } else if (found != 1 && emit_phase_block<Real>(ops, rest, ro, R, loc_of, tmask, 2, out)) {
            continue;
        } else if (emit_xset<Real>(ops, rest, ro, loc_of, tmask, out)) {
            // relabeling X gates as late as the schedule allows: fewer later
            // gates see a relabeled bit
            continue;
        } else {
            out.push_back(encode<Real>(ops[rest[0]], ro, loc_of, tmask));
            keep.assign(rest.begin() + 1, rest.end());
        }
        rest.swap(keep);
    }
}

template <typename Real>
SmallOp<Real> encode_small(const SOp &o) {
    SmallOp<Real> s;
    memset(&s, 0, sizeof s);
    s.target = o.target;
    s.kind = o.mc;
    s.cmask = (uint32_t)o.cmask;
    s.cval = (uint32_t)o.cval;
    for (int k = 0; k < 4; k++) {
        s.m[2 * k] = (Real)o.m[k].real();
        s.m[2 * k + 1] = (Real)o.m[k].imag();
    }
    return s;
}

// Doubly linked list over op indices (scheduling removes from the middle).
struct OpList {
    std::vector<int> nxt, prv;
    int head = -1;
    explicit OpList(int n) : nxt(n), prv(n) {
        for (int i = 0; i < n; i++) {
            nxt[i] = i + 1 < n ? i + 1 : -1;
            prv[i] = i - 1;
        }
        head = n ? 0 : -1;
    }
    void remove(int i) {
        if (prv[i] >= 0) nxt[prv[i]] = nxt[i];
        else head = nxt[i];
        if (nxt[i] >= 0) prv[nxt[i]] = prv[i];
    }
};

// Whether the encoded op records need only the pass kernel's lean build
// (Plan::lean): phase blocks of compact terms, real and split layers,
// relabeling X records, and on register bits only diagonal, phase and X
// gates.
template <typename Real>
bool lean_ops(const std::vector<DevOp<Real>> &d, int R) {
    for (size_t i = 0; i < d.size();) {
        const DevOp<Real> &o = d[i];
        switch (o.kind) {
            case K_PHASE_BLOCK:
                if (!(o.cm_reg & PB_ANGLES)) return false;
                i += 1 + (size_t)o.tpos;
                break;
            case K_LAYER:
                return false;
            case K_LAYER_REAL:
            case K_LAYER_SPLIT:
                i += 1 + (size_t)__builtin_popcount(o.cm_reg);
                break;
            case K_DENSE:
            case K_REAL:
            case K_ANTI:
                if (o.tpos < R) return false;
                i++;
                break;
            default:
                i++;
        }
    }
    return true;
}

template <typename Real>
int build_tiled(const std::vector<SOp> &ops, int n, const hgm_plan_opts &o, Plan *plan) {
    const int W = plan->warp_bits;
    const int R = plan->reg_bits;
    const int K = 5 + R + W;
    const int L = std::min(o.low_bits, K);
    const int window = o.window > 0 ? o.window : 4096;
    const uint64_t all_bits = (n >= 64) ? ~uint64_t(0) : ((uint64_t(1) << n) - 1);
    std::vector<DevOp<Real>> dev_ops;
    dev_ops.reserve(ops.size());
    const LayoutMaker lm{R, W, K, sizeof(Real) == 8 ? 3 : 4, L};
    auto intern = [&](const Lay &lay) {
        for (size_t i = 0; i < plan->layouts.size(); i++)
            if (!memcmp(plan->layouts[i].pos, lay.pos, sizeof lay.pos)) return (int)i;
        plan->layouts.push_back(lay);
        return (int)plan->layouts.size() - 1;
    };

    // product of the scalars split layers leave out (emit_phase)
    cplx global = 1.0;
    OpList list((int)ops.size());
    std::vector<int> pass_ops;
    int pass_index = 0;
    while (list.head >= 0) {
        uint64_t tmask = (uint64_t(1) << L) - 1;
        int tcount = L;
        uint64_t b_nd = 0, b_d = 0;
        pass_ops.clear();
        int since_take = 0;
        for (int i = list.head; i >= 0;) {
            const SOp &op = ops[i];
            int nexti = list.nxt[i];
            bool take = false;
            if (!conflicts(op, b_nd, b_d)) {
                uint64_t tb = uint64_t(1) << op.target;
                if (op.mc == MC_DIAG || (tmask & tb)) take = true;
                else if (tcount < K) {
                    tmask |= tb;
                    tcount++;
                    take = true;
                }
            }
            if (take) {
                pass_ops.push_back(i);
                list.remove(i);
                since_take = 0;
            } else {
                b_nd |= op.nd();
                b_d |= op.dg();
                if (++since_take > window) break;
                if ((b_nd & all_bits) == all_bits) break;
            }
            i = nexti;
        }
        if (pass_ops.empty()) return fail(HGM_ERR_INVALID, "planner made no progress");
        // fill the tile up to K bits with the lowest unused index bits
        for (int g = 0; tcount < K && g < n; g++) {
            if (!((tmask >> g) & 1)) {
                tmask |= uint64_t(1) << g;
                tcount++;
            }
        }
        // local positions: the low bits at local 0..L-1; the others by first
        // dense use at local 5 and up, then the lane bits above L
        std::vector<int> order;
        uint64_t placed = (uint64_t(1) << L) - 1;
        for (int idx : pass_ops) {
            const SOp &op = ops[idx];
            uint64_t tb = uint64_t(1) << op.target;
            if (op.mc != MC_DIAG && !(placed & tb)) {
                placed |= tb;
                order.push_back(op.target);
            }
        }
        for (int g = 0; g < n; g++)
            if (((tmask >> g) & 1) && !((placed >> g) & 1)) {
                placed |= uint64_t(1) << g;
                order.push_back(g);
            }
        std::vector<int> slots;
        for (int q = 5; q < 5 + R; q++) slots.push_back(q);
        for (int q = 5 + R; q < 5 + R + W; q++) slots.push_back(q);
        if (R == 4 && L <= 4) slots.push_back(4);
        for (int q = L; q < R; q++) slots.push_back(q);
        int loc_of[64];
        for (int g = 0; g < 64; g++) loc_of[g] = -1;
        PassArgs pa;
        memset(&pa, 0, sizeof pa);
        pa.n = n;
        pa.k = K;
        for (int g = 0; g < L; g++) {
            loc_of[g] = g;
            pa.tb[g] = (int8_t)g;
        }
        for (size_t j = 0; j < order.size(); j++) {
            loc_of[order[j]] = slots[j];
            pa.tb[slots[j]] = (int8_t)order[j];
        }
        pa.tile_mask = tmask;
        for (int g = 0; g < n;) {
            if ((tmask >> g) & 1) {
                g++;
                continue;
            }
            int e = g;
            while (e < n && !((tmask >> e) & 1)) e++;
            pa.run_pos[pa.nruns] = (int8_t)g;
            pa.run_len[pa.nruns] = (int8_t)(e - g);
            pa.nruns++;
            g = e;
        }

        // register phases: each takes the gates that can move to the front
        // with their targets on its register bits.  A phase keeps the
        // previous layout unless a new register set, chosen first-fit from
        // the pending gates, takes more of them.
        pa.phase_begin = (int)plan->phases.size();
        std::vector<int> pending = pass_ops;
        int cur = -1;
        std::vector<int> taken, rest;
        auto walk = [&](uint32_t S, std::vector<int> *tk, std::vector<int> *rs) {
            uint64_t bn = 0, bd = 0;
            int count = 0;
            for (int idx : pending) {
                const SOp &op = ops[idx];
                bool ok = !conflicts(op, bn, bd) && (op.mc == MC_DIAG || ((S >> loc_of[op.target]) & 1));
                if (ok) {
                    count++;
                    if (tk) tk->push_back(idx);
                } else {
                    if (rs) rs->push_back(idx);
                    bn |= op.nd();
                    bd |= op.dg();
                }
            }
            return count;
        };
        // low_first: a first walk lets only gates on the low index bits
        // (local 0..L-1) claim register bits, so that a phase needing them
        // comes while later phases can still end the pass in a coalesced
        // layout (a low-bit phase left last costs a store transpose)
        auto first_fit = [&](uint32_t prefer, bool low_first) {
            uint32_t S = 0;
            for (int round = low_first ? 0 : 1; round < 2; round++) {
                uint64_t bn = 0, bd = 0;
                for (int idx : pending) {
                    const SOp &op = ops[idx];
                    bool ok = !conflicts(op, bn, bd);
                    if (ok && op.mc != MC_DIAG) {
                        const int l = loc_of[op.target];
                        const uint32_t b = 1u << l;
                        if (!(S & b)) {
                            if (round == 0 && l >= L) ok = false;
                            else if (__builtin_popcount(S) < R && lm.feasible(S | b)) S |= b;
                            else ok = false;
                        }
                    }
                    if (!ok) {
                        bn |= op.nd();
                        bd |= op.dg();
                    }
                }
            }
            return lm.fill(S, prefer);
        };
        while (!pending.empty()) {
            const uint32_t cur_S = cur >= 0 ? LayoutMaker::regs(plan->layouts[cur], R, W) : 0;
            const int count_cur = cur >= 0 ? walk(cur_S, nullptr, nullptr) : -1;
            const uint32_t S_new = first_fit(cur_S, cur >= 0);
            const int count_new = walk(S_new, nullptr, nullptr);
            int lay = cur;
            uint32_t S = cur_S;
            if (cur < 0 || count_new > count_cur) {
                S = S_new;
                lay = intern(lm.make(S, cur >= 0 ? &plan->layouts[cur] : nullptr));
            }
            taken.clear();
            rest.clear();
            walk(S, &taken, &rest);
            if (taken.empty()) return fail(HGM_ERR_INVALID, "phase scheduling made no progress");
            DevPhase ph;
            ph.layout = lay;
            ph.op_begin = (int)dev_ops.size();
            Roles ro(plan->layouts[lay], R, W);
            for (int t = 0; t < 5 + W; t++) ro.thr_gbit[t] = pa.tb[plan->layouts[lay].pos[t]];
            emit_phase<Real>(ops, taken, ro, R, loc_of, tmask, o.split_layers != 0, global, dev_ops);
            ph.op_end = (int)dev_ops.size();
            ph.xwarp = 0;
            if (cur >= 0 && cur != lay) {
                ph.xwarp = lm.same_warps(plan->layouts[cur], plan->layouts[lay]) ? 0 : 1;
                plan->n_transposes++;
            }
            plan->phases.push_back(ph);
            cur = lay;
            pending.swap(rest);
        }
        pa.phase_end = (int)plan->phases.size();
        // load and store layouts: the first and last phase's when coalesced,
        // else one with the same warp bits and no low index bit in registers
        DevPhase &first = plan->phases[pa.phase_begin];
        pa.load_layout = first.layout;
        if (!lm.coalesced(plan->layouts[first.layout])) {
            const Lay f = plan->layouts[first.layout];
            const uint32_t avoid = (1u << L) - 1;
            uint32_t S0 = lm.fill(LayoutMaker::regs(f, R, W) & ~avoid, 0);
            pa.load_layout = intern(lm.make(S0, &f));
            first.xwarp = lm.same_warps(plan->layouts[pa.load_layout], f) ? 0 : 1;
            plan->n_transposes++;
        }
        pa.store_layout = cur;
        pa.store_xwarp = 0;
        if (!lm.coalesced(plan->layouts[cur])) {
            const Lay c = plan->layouts[cur];
            const uint32_t avoid = (1u << L) - 1;
            uint32_t S1 = lm.fill(LayoutMaker::regs(c, R, W) & ~avoid, 0);
            pa.store_layout = intern(lm.make(S1, &c));
            pa.store_xwarp = lm.same_warps(plan->layouts[pa.store_layout], c) ? 0 : 1;
            plan->n_transposes++;
        }
        for (int k = 0; k < 5 + W + R; k++) {
            pa.ld_gbit[k] = pa.tb[plan->layouts[pa.load_layout].pos[k]];
            pa.st_gbit[k] = pa.tb[plan->layouts[pa.store_layout].pos[k]];
        }
        plan->passes.push_back(pa);
        pass_index++;
    }
    if (global != 1.0) {
        // the split layers' scalars, once at the end: diag(g, g) on register bit 0
        DevOp<Real> d;
        memset(&d, 0, sizeof d);
        d.kind = K_DIAG;
        d.m[0] = d.m[6] = (Real)global.real();
        d.m[1] = d.m[7] = (Real)global.imag();
        dev_ops.push_back(d);
        plan->phases.back().op_end = (int)dev_ops.size();
    }
    plan->lean = lean_ops<Real>(dev_ops, R);
    plan->ops_bytes.resize(dev_ops.size() * sizeof(DevOp<Real>));
    if (!dev_ops.empty()) memcpy(plan->ops_bytes.data(), dev_ops.data(), plan->ops_bytes.size());
    return HGM_OK;
}

template <typename Real>
int build_small(const std::vector<SOp> &ops, Plan *plan) {
    std::vector<SmallOp<Real>> so;
    so.reserve(ops.size());
    for (const SOp &o : ops) so.push_back(encode_small<Real>(o));
    plan->ops_bytes.resize(so.size() * sizeof(SmallOp<Real>));
    if (!so.empty()) memcpy(plan->ops_bytes.data(), so.data(), plan->ops_bytes.size());
    plan->n_small_ops = (int64_t)so.size();
    return HGM_OK;
}

}  // namespace

int build_plan(const std::vector<Op> &ops, int n, const hgm_plan_opts &opts, Plan *plan, bool force_small) {
    if (n < 1 || n > 34) return fail(HGM_ERR_UNSUPPORTED, "qubits=%d outside 1..34", n);
    for (const Op &op : ops) {
        if (op.target < 0 || op.target >= n) return fail(HGM_ERR_INVALID, "target bit %d outside 0..%d", op.target, n - 1);
        if (n < 64 && (op.cmask >> n)) return fail(HGM_ERR_INVALID, "control mask beyond %d qubits", n);
        if (op.cmask & (uint64_t(1) << op.target)) return fail(HGM_ERR_INVALID, "target is also a control");
    }
    plan->precision = opts.precision;
    plan->qubits = n;
    plan->renorm_every = opts.precision == HGM_F32 ? opts.renorm_every : 0;
    plan->chained = opts.chained != 0;
    std::vector<SOp> sops = fuse_ops(ops, opts.fuse);
    plan->n_ops = (int64_t)sops.size();
    // amplitudes per thread: 16 for FP64 (64 data registers), 32 for FP32
    // (or 16 on request: plan_reg_bits)
    const int R = plan_reg_bits(opts.precision, n, opts.reg_bits);
    if (R < 0) return fail(HGM_ERR_INVALID, "reg_bits=%d not available for this precision", opts.reg_bits);
    plan->reg_bits = R;
    if (n < 5 + R || force_small) {
        if (n > 14) return fail(HGM_ERR_UNSUPPORTED, "the shared-memory path takes at most 14 qubits");
        plan->small = true;
        plan->warp_bits = 0;
        return opts.precision == HGM_F64 ? build_small<double>(sops, plan) : build_small<float>(sops, plan);
    }
    // Default CTA: 4 warps (tile of 2^11 FP64 / 2^12 FP32 amplitudes), the
    // fastest size in the pass micro-benchmarks for both precisions.
    int W = opts.warp_bits;
    if (W < 0) W = 2;
    W = std::min(W, 3);
    W = std::min(W, n - 5 - R);
    plan->warp_bits = W;
    hgm_plan_opts o = opts;
    if (o.low_bits < 0) o.low_bits = opts.precision == HGM_F64 ? 3 : 4;
    o.low_bits = std::max(0, std::min(o.low_bits, 5));
    return opts.precision == HGM_F64 ? build_tiled<double>(sops, n, o, plan) : build_tiled<float>(sops, n, o, plan);
}

}  // namespace hgm
