"""CPU emulation of a plan's encoded passes (test helper).

Re-executes, with numpy, exactly what the pass kernel (simulador_quantico_b200/
csrc/kernels.cuh) does with a plan's encoding: per pass, every tile of 2^K
amplitudes is gathered through the tile-bit map, the register phases run
with their layout's (lane, warp, register) coordinates and the encoded
controls, and the tile is scattered back.  Comparing its result with the
oracle checks the planner and the encoding without a GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from simulador_quantico_b200._lib import check, lib

PASS_DT = np.dtype([("n", "<i4"), ("k", "<i4"), ("phase_begin", "<i4"), ("phase_end", "<i4"),
                    ("load_layout", "<i4"), ("store_layout", "<i4"), ("flags", "<i4"), ("store_xwarp", "<i4"),
                    ("tb", "i1", 16), ("tile_mask", "<u8"), ("phases", "<u8"), ("ops", "<u8"),
                    ("norm_out", "<u8"), ("scale_in", "<u8"), ("layouts", "<u8"), ("run_pos", "i1", 18),
                    ("run_len", "i1", 18), ("nruns", "<i4"), ("ld_gbit", "i1", 16), ("st_gbit", "i1", 16)])
PHASE_DT = np.dtype([("layout", "<i4"), ("op_begin", "<i4"), ("op_end", "<i4"), ("xwarp", "<i4")])


def op_dtype(real):
    fields = [("kind", "<i4"), ("tpos", "<i4"), ("cm_reg", "<u4"), ("cv_reg", "<u4"), ("cm_thr", "<u4"),
              ("cv_thr", "<u4"), ("tpos2", "<i4"), ("pad1", "<u4"), ("cm_glob", "<u8"), ("cv_glob", "<u8"),
              ("m", real, 8)]
    dt = np.dtype(fields)
    size = (dt.itemsize + 15) // 16 * 16
    return np.dtype({"names": dt.names, "formats": [dt.fields[n][0] for n in dt.names],
                     "offsets": [dt.fields[n][1] for n in dt.names], "itemsize": size})


SMALL_DT = {"<f8": np.dtype([("target", "<i4"), ("kind", "<i4"), ("cmask", "<u4"), ("cval", "<u4"), ("m", "<f8", 8)]),
            "<f4": np.dtype([("target", "<i4"), ("kind", "<i4"), ("cmask", "<u4"), ("cval", "<u4"), ("m", "<f4", 8)])}

K_DENSE, K_REAL, K_DIAG, K_PHASE, K_ANTI, K_SWAP, K_LAYER, K_LAYER_REAL, K_PHASE_BLOCK, K_LAYER_SPLIT, K_XSET = range(11)
XSET_CTRL_NONE, XSET_CTRL_THREAD, XSET_CTRL_GLOBAL = 0, 2, 3
PB_F_ACTIVE = 1 << 16
REG_BITS = {"f64": 4, "f32": 5}
PB_LINEAR = -2  # hgm_internal.h: a linear phase term
PB_GATED, PB_GATE_SHIFT = 4, 8  # hgm_internal.h: a phase block gated by one register bit


def export(plan, precision):
    p, np_, ph, nph, ops, nb = C.c_void_p(), C.c_int64(), C.c_void_p(), C.c_int64(), C.c_void_p(), C.c_int64()
    wb, sm = C.c_int(), C.c_int()
    check(lib.hgm_plan_export(plan.h, C.byref(p), C.byref(np_), C.byref(ph), C.byref(nph), C.byref(ops), C.byref(nb),
                              C.byref(wb), C.byref(sm)))
    real = "<f8" if precision == "f64" else "<f4"
    passes = np.frombuffer(C.string_at(p, np_.value * PASS_DT.itemsize), PASS_DT) if np_.value else np.zeros(0, PASS_DT)
    phases = np.frombuffer(C.string_at(ph, nph.value * PHASE_DT.itemsize), PHASE_DT) if nph.value else np.zeros(0, PHASE_DT)
    raw = C.string_at(ops, nb.value) if nb.value else b""
    odt = SMALL_DT[real] if sm.value else op_dtype(real)
    opsarr = np.frombuffer(raw, odt) if raw else np.zeros(0, odt)
    lp, nl = C.c_void_p(), C.c_int64()
    check(lib.hgm_plan_layouts(plan.h, C.byref(lp), C.byref(nl)))
    layouts = (np.frombuffer(C.string_at(lp, nl.value * 16), np.int8).reshape(nl.value, 16).astype(np.int64)
               if nl.value else np.zeros((0, 16), np.int64))
    return dict(passes=passes, phases=phases, ops=opsarr, W=wb.value, small=bool(sm.value), layouts=layouts)


def layout_coords(pos, R, W, K):
    """For every local index j: (lane, warp, reg) in the layout whose roles
    (thread bits 0..4+W, then register bits) sit on local bits pos[...]."""
    j = np.arange(1 << K)
    thr = sum(((j >> int(pos[t])) & 1) << t for t in range(5 + W))
    reg = sum(((j >> int(pos[5 + W + q])) & 1) << q for q in range(R))
    return thr & 31, thr >> 5, reg


def local_of(pos, R, W, lane, warp, reg):
    thr = lane | (warp << 5)
    j = sum(((thr >> t) & 1) << int(pos[t]) for t in range(5 + W))
    return j | sum(((reg >> q) & 1) << int(pos[5 + W + q]) for q in range(R))


def check_pass_layouts(e, pa, R, W, K, low_bits=3):
    """The kernel's assumptions about a pass's layouts: every layout is a
    permutation of the K local bits; its low thread bits keep the padded
    transposes free of bank conflicts; the load and store layouts move whole
    runs of the low index bits; the global bits handed to the kernel match;
    a transpose marked warp-local keeps every warp bit in place."""
    nb = 3 if R == 4 else 4
    per = {"<f8": 8, "<f4": 16}
    lays = e["layouts"]
    phases = e["phases"][pa["phase_begin"]:pa["phase_end"]]
    used = {int(pa["load_layout"]), int(pa["store_layout"])} | {int(ph["layout"]) for ph in phases}
    for li in used:
        pos = lays[li][:5 + W + R]
        assert sorted(pos.tolist()) == list(range(K)), pos
        slots = {sum(((lane >> t) & 1) * ((1 << int(pos[t])) + ((1 << int(pos[t])) >> R)) for t in range(nb))
                 % (1 << nb) for lane in range(1 << nb)}
        assert len(slots) == 1 << nb, ("bank conflict", pos)
    tb = [int(x) for x in pa["tb"][:K]]
    for key, li in (("ld_gbit", int(pa["load_layout"])), ("st_gbit", int(pa["store_layout"]))):
        pos = lays[li]
        assert [int(x) for x in pa[key][:5 + W + R]] == [tb[int(pos[k])] for k in range(5 + W + R)]
        # the planner keeps index bits 0..low_bits-1 at local 0..low_bits-1
        # and puts them on thread bits 0..low_bits-1 of these layouts
        for t in range(min(low_bits, 5, K)):
            assert tb[t] == t and int(pos[t]) == t, ("uncoalesced", key, pos)
    cur = int(pa["load_layout"])

    def same_warps(a, b):
        return all(lays[a][5 + w] == lays[b][5 + w] for w in range(W))
    for ph in phases:
        if int(ph["layout"]) != cur and not int(ph["xwarp"]):
            assert same_warps(cur, int(ph["layout"]))
        cur = int(ph["layout"])
    if cur != int(pa["store_layout"]) and not int(pa["store_xwarp"]):
        assert same_warps(cur, int(pa["store_layout"]))


def apply_small(state, ops, n):
    N = 1 << n
    idx = np.arange(N)
    for o in ops:
        t, cm, cv = int(o["target"]), int(o["cmask"]), int(o["cval"])
        m = o["m"].astype(np.float64)
        mm = m[0::2] + 1j * m[1::2]
        i0 = idx[((idx >> t) & 1) == 0]
        i0 = i0[(i0 & cm) == cv]
        i1 = i0 | (1 << t)
        a0, a1 = state[i0].copy(), state[i1].copy()
        state[i0] = mm[0] * a0 + mm[1] * a1
        state[i1] = mm[2] * a0 + mm[3] * a1
    return state


def apply_reg_pair(tile, lay, R, W, lane, warp, reg, tpos, ok_t, ok_j, kind, mm):
    bit = (reg >> tpos) & 1
    sel = np.nonzero((bit == 0) & ok_j)[0]
    partner = local_of(lay, R, W, lane[sel], warp[sel], reg[sel] | (1 << tpos))
    rows = np.nonzero(ok_t)[0]
    a0 = tile[np.ix_(rows, sel)]
    a1 = tile[np.ix_(rows, partner)]
    if kind == K_SWAP:
        n0, n1 = a1, a0
    elif kind == K_ANTI:
        n0, n1 = mm[1] * a1, mm[2] * a0
    else:
        n0, n1 = mm[0] * a0 + mm[1] * a1, mm[2] * a0 + mm[3] * a1
    tile[np.ix_(rows, sel)] = n0
    tile[np.ix_(rows, partner)] = n1
    return tile


def _term_factor(t, base, thr):
    """Per (tile, thread) factor of one phase-block term and whether it applies: arrays [T, nthr]."""
    m = t["m"].astype(np.float64)
    d0, d1 = m[0] + 1j * m[1], m[6] + 1j * m[7]
    ok = ((base & int(t["cm_glob"])) == int(t["cv_glob"]))[:, None] & ((thr & int(t["cm_thr"])) == int(t["cv_thr"]))[None, :]
    tpos = int(t["tpos"])
    if tpos >= 64:
        bv = ((base >> (tpos - 64)) & 1)[:, None] * np.ones_like(thr)[None, :]
    elif tpos >= 8:
        bv = np.broadcast_to(((thr >> (tpos - 8)) & 1)[None, :], ok.shape)
    else:
        bv = np.zeros(ok.shape, dtype=np.int64)
    f0 = np.where(bv == 1, d1, d0)
    return ok, f0, d1


def phase_terms(recs, first, count, real):
    """The compact phase terms (struct PhaseTerm) packed in records first.. :
    a list of (cbit, cval, tbit, a0, a1)."""
    size = 16 if real == "<f4" else 32
    per = recs.dtype.itemsize // size
    tdt = np.dtype([("cbit", "i1"), ("cval", "i1"), ("tbit", "i1"), ("pad", "i1", size // 4 - 3),
                    ("a0", real), ("a1", real), ("pad2", real)])
    out = []
    for k in range(count):
        raw = recs[first + k // per].tobytes()[(k % per) * size:(k % per + 1) * size]
        t = np.frombuffer(raw, tdt)[0]
        if int(t["cbit"]) == PB_LINEAR:
            # linear term: mask where a0 (and a1 in FP32) sit, scale in pad2 (FP32) or a1 (FP64)
            rs = size // 4
            mask = int.from_bytes(raw[rs:rs + 8], "little")
            scale = float(np.frombuffer(raw[3 * rs:4 * rs] if size == 16 else raw[2 * rs:3 * rs], real)[0])
            out.append(("linear", int(t["cval"]) & 1, int(t["tbit"]), mask, scale))
        else:
            out.append((int(t["cbit"]), int(t["cval"]), int(t["tbit"]), float(t["a0"]), float(t["a1"])))
    return out


def linear_value(ix, rev, mask, scale):
    """A linear term's turns: scale times the masked index, or with rev the
    masked bits weighted 2^-b."""
    if not rev:
        return scale * (ix & mask).astype(np.float64)
    v = np.zeros(ix.shape)
    for b in range(64):
        if (mask >> b) & 1:
            v += ((ix >> b) & 1) * 2.0 ** (-b)
    return scale * v


def apply_phase_block_angles(tile, recs, i, R, base, thr, reg, T, K, real):
    """A phase block of compact phase terms (head flag PB_ANGLES): phases add
    up in turns per category; the kernel folds F into the first active bit."""
    head = recs[i]
    counts = np.frombuffer(head["m"].tobytes()[:16], dtype=np.uint8)
    tgb = np.frombuffer(head["m"].tobytes()[16:24], dtype=np.int8)
    has_table = int(head["cm_reg"]) & 1
    act = int(head["cv_reg"])
    nrec = int(head["tpos"])
    ix = base[:, None] | np.zeros((1, 1 << K), dtype=np.int64)
    for t in range(8):
        ix = ix | (((thr >> t) & 1).astype(np.int64) << int(tgb[t]))[None, :]
    terms = phase_terms(recs, i + 1, int(sum(int(c) for c in counts)), real)
    if int(head["cm_reg"]) & PB_GATED:
        # the kernel's gated form multiplies only the registers whose label bit
        # g is 1: every other factor of the block must be exactly 1
        g = (int(head["cm_reg"]) >> PB_GATE_SHIFT) & 7
        assert has_table  # the kernel's gated sweep always reads a table
        assert all(int(c) == 0 for k, c in enumerate(counts) if k not in (1 + g, 1 + 2 * R + g)), counts
        for t in terms[int(counts[1 + g]):]:
            assert t[0] == "linear" or t[3] == 0.0, t
        if has_table:
            j = i + 1 + nrec - (1 << R) // 4
            tab = np.concatenate([recs[j + q]["m"].astype(np.float64) for q in range((1 << R) // 4)])
            tab = tab[0::2] + 1j * tab[1::2]
            assert all(tab[r] == 1.0 for r in range(1 << R) if not (r >> g) & 1)
    phase = np.zeros((T, 1 << K))

    def contrib(term):
        if term[0] == "linear":
            _, rev, tbit, mask, scale = term
            c = np.ones(ix.shape, bool) if tbit < 0 else (((ix >> tbit) & 1) == 1)
            return c, linear_value(ix, rev, mask, scale)
        cbit, cval, tbit, a0, a1 = term
        c = np.ones(ix.shape, bool) if cbit < 0 else (((ix >> cbit) & 1) == cval)
        t = np.zeros(ix.shape, np.int64) if tbit < 0 else ((ix >> tbit) & 1)
        return c, np.where(t == 1, a1, a0)
    k = 0
    for _ in range(int(counts[0])):
        c, a = contrib(terms[k])
        if act & PB_F_ACTIVE:
            phase += np.where(c, a, 0.0)
        k += 1
    for b in range(R):
        bit = ((reg >> b) & 1)[None, :]
        for kind, cnt in (("G", counts[1 + b]), ("H", counts[1 + R + b]), ("D", counts[1 + 2 * R + b])):
            for _ in range(int(cnt)):
                if (act >> b) & 1:
                    c, a = contrib(terms[k])
                    if kind == "G":
                        phase += np.where(c & (bit == 1), a, 0.0)
                    elif kind == "H":
                        phase += np.where(c & (bit == 0), a, 0.0)
                    elif terms[k][0] == "linear":  # a D term folded: adds where the register bit is 1
                        phase += np.where(c & (bit == 1), a, 0.0)
                    else:
                        cbit, cval, tbit, a0, a1 = terms[k]
                        phase += np.where(c, np.where(bit == 1, a1, a0), 0.0)
                k += 1
    f = np.exp(2j * np.pi * phase)
    if has_table:
        j = i + 1 + nrec - (1 << R) // 4
        tab = []
        for q in range((1 << R) // 4):
            m = recs[j + q]["m"].astype(np.float64)
            tab += list(m[0::2] + 1j * m[1::2])
        f = f * np.asarray(tab)[reg][None, :]
    return tile * f


def apply_phase_block(tile, recs, i, R, base, thr, reg, T, K, real="<f8"):
    if int(recs[i]["cm_reg"]) & 2:
        return apply_phase_block_angles(tile, recs, i, R, base, thr, reg, T, K, real)
    counts = np.frombuffer(recs[i]["m"].tobytes()[:16], dtype=np.uint8)
    has_table = int(recs[i]["cm_reg"]) & 1
    act = int(recs[i]["cv_reg"])  # active register bits; PB_F_ACTIVE: F terms
    j = i + 1
    f = np.ones((T, 1 << K), dtype=np.complex128)
    for _ in range(int(counts[0])):
        ok, f0, _d1 = _term_factor(recs[j], base, thr)
        if act & PB_F_ACTIVE:
            f = np.where(ok, f * f0, f)
        j += 1
    for b in range(R):
        bit = ((reg >> b) & 1)[None, :]
        for kind, cnt in (("G", counts[1 + b]), ("H", counts[1 + R + b]), ("D", counts[1 + 2 * R + b])):
            for _ in range(int(cnt)):
                if not (act >> b) & 1:  # the kernel skips an inactive bit's terms
                    j += 1
                    continue
                ok, f0, d1 = _term_factor(recs[j], base, thr)
                if kind == "G":
                    fac = np.where(bit == 1, f0, 1.0)
                elif kind == "H":
                    fac = np.where(bit == 0, f0, 1.0)
                else:
                    fac = np.where(bit == 1, d1, f0)
                f = np.where(ok, f * fac, f)
                j += 1
    if has_table:
        tab = []
        for q in range((1 << R) // 4):
            m = recs[j + q]["m"].astype(np.float64)
            tab += list(m[0::2] + 1j * m[1::2])
        f = f * np.asarray(tab)[reg][None, :]
    return tile * f


def run(plan, precision, state, iterations=1):
    e = export(plan, precision)
    n = plan.qubits
    state = np.asarray(state, dtype=np.complex128).copy()
    if e["small"]:
        for _ in range(iterations):
            apply_small(state, e["ops"], n)
        return state
    W = e["W"]
    for _ in range(iterations):
        for pa in e["passes"]:
            K = int(pa["k"])
            R = K - 5 - W  # the plan's register bits (FP32: 4 or 5)
            lb = getattr(getattr(plan, "opts", None), "low_bits", -1)
            if lb < 0:
                lb = 3 if precision == "f64" else 4
            check_pass_layouts(e, pa, R, W, K, lb)
            tb = [int(x) for x in pa["tb"][:K]]
            tmask = int(pa["tile_mask"])
            free = [g for g in range(n) if not (tmask >> g) & 1]
            T = 1 << len(free)
            tiles = np.arange(T, dtype=np.int64)
            base = np.zeros(T, dtype=np.int64)
            for k, g in enumerate(free):
                base |= ((tiles >> k) & 1) << g
            # the kernels deposit the tile number run by run
            runs, shift = np.zeros(T, dtype=np.int64), 0
            for i in range(int(pa["nruns"])):
                ln, pos = int(pa["run_len"][i]), int(pa["run_pos"][i])
                runs |= ((tiles >> shift) & ((1 << ln) - 1)) << pos
                shift += ln
            assert shift == len(free) and np.array_equal(runs, base)
            j = np.arange(1 << K, dtype=np.int64)
            scat = np.zeros(1 << K, dtype=np.int64)
            for q, g in enumerate(tb):
                scat |= ((j >> q) & 1) << g
            gidx = base[:, None] | scat[None, :]
            tile = state[gidx]  # [T, 2^K] by local index
            for ph in e["phases"][pa["phase_begin"]:pa["phase_end"]]:
                lay = e["layouts"][int(ph["layout"])]
                lane, warp, reg = layout_coords(lay, R, W, K)
                thr = lane | (warp << 5)
                recs = e["ops"][ph["op_begin"]:ph["op_end"]]
                i = 0
                while i < len(recs):
                    o = recs[i]
                    if int(o["kind"]) == K_PHASE_BLOCK:
                        tile = apply_phase_block(tile, recs, i, R, base, thr, reg, T, K,
                                                 "<f8" if precision == "f64" else "<f4")
                        i += 1 + int(o["tpos"])
                        continue
                    if int(o["kind"]) == K_XSET:
                        # relabeling X gates: target register bit, control on a thread or non-tile bit
                        ent = np.frombuffer(o["m"].tobytes(), np.uint8).reshape(-1, 4)[:int(o["tpos"])]
                        for t, ck, cb, cv in ent.astype(np.int64):
                            ok_t = np.ones(T, bool)
                            ok_j = np.ones(1 << K, bool)
                            if ck == XSET_CTRL_THREAD:
                                ok_j = ((thr >> cb) & 1) == cv
                            elif ck == XSET_CTRL_GLOBAL:
                                ok_t = ((base >> cb) & 1) == cv
                            else:
                                assert ck == XSET_CTRL_NONE and cv == 0
                            tile = apply_reg_pair(tile, lay, R, W, lane, warp, reg, int(t), ok_t, ok_j, K_SWAP, None)
                        i += 1
                        continue
                    if int(o["kind"]) in (K_LAYER, K_LAYER_REAL, K_LAYER_SPLIT):
                        # uncontrolled dense gates on the register bits of the mask, lowest first
                        mask = int(o["cm_reg"])
                        k = 0
                        for t in range(R):
                            if not (mask >> t) & 1:
                                continue
                            mm = recs[i + 1 + k]["m"].astype(np.float64)
                            if int(o["kind"]) == K_LAYER_SPLIT:
                                # Rm diag(1, p): Rm real in m[0..3], p in m[4..5]
                                flags = int(o["cv_reg"])
                                p = mm[4] + 1j * mm[5] if (flags >> t) & 1 else 1.0
                                mm = np.array([mm[0], mm[1] * p, mm[2], mm[3] * p], dtype=np.complex128)
                            else:
                                mm = mm[0::2] + 1j * mm[1::2]
                            tile = apply_reg_pair(tile, lay, R, W, lane, warp, reg, t, np.ones(T, bool),
                                                  np.ones(1 << K, bool), K_DENSE, mm)
                            k += 1
                        i += 1 + k
                        continue
                    i += 1
                    m = o["m"].astype(np.float64)
                    mm = m[0::2] + 1j * m[1::2]
                    kind, tpos = int(o["kind"]), int(o["tpos"])
                    ok_t = (base & int(o["cm_glob"])) == int(o["cv_glob"])           # [T]
                    ok_j = ((thr & int(o["cm_thr"])) == int(o["cv_thr"])) & ((reg & int(o["cm_reg"])) == int(o["cv_reg"]))
                    if tpos < R:
                        bit = (reg >> tpos) & 1
                        if kind in (K_DIAG, K_PHASE):
                            f = np.where(bit == 1, mm[3], mm[0] if kind == K_DIAG else 1.0)
                            mask = ok_t[:, None] & ok_j[None, :]
                            tile = np.where(mask, tile * f[None, :], tile)
                        else:
                            tile = apply_reg_pair(tile, lay, R, W, lane, warp, reg, tpos, ok_t, ok_j, kind, mm)
                    else:
                        if tpos >= 64:
                            bv = ((base >> (tpos - 64)) & 1)[:, None] * np.ones((1, 1 << K), dtype=np.int64)
                        else:
                            bv = np.broadcast_to(((thr >> (tpos - 8)) & 1)[None, :], (T, 1 << K))
                        f = np.where(bv == 1, mm[3], mm[0] if kind == K_DIAG else 1.0)
                        mask = ok_t[:, None] & ok_j[None, :]
                        tile = np.where(mask, tile * f, tile)
            state[gidx] = tile
    return state
