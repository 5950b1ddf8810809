// Host mirror of the reference's circuit language and gate catalogue.
//
// Parses gate strings into the op list exactly as the reference's DGM does
// (MMullerdR/simulador_quantico):
//   Tokenize              src/core/dgm_parser.cpp:10-26
//   DGM::setFunction      src/core/dgm_parser.cpp:29-66 (unroll, per-step sort)
//   DGM::genGroups        src/core/dgm_parser.cpp:70-114
//   DGM::genPTs           src/core/dgm_parser.cpp:118-169
//   increasing/decreasing src/core/common.cpp:166-178
//   Gates::init/addGate   src/core/gates.cpp:23-60
// Gate matrices are computed and stored in FP64 (the FP32 engine casts them),
// where the reference builds them in FP32 with cpowf.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "hgm_dropin_layout.h"
#include "hgm_internal.h"

namespace hgm {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

int fail(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

MatClass classify(const cplx m[4]) {
    if (m[1] == 0.0 && m[2] == 0.0) return MC_DIAG;
    if (m[0] == 0.0 && m[3] == 0.0) return MC_ANTI;
    return MC_DENSE;
}

static void tokenize(const std::string &text, std::vector<std::string> &out, const char *delims) {
    std::string::size_type last = text.find_first_not_of(delims, 0);
    std::string::size_type pos = text.find_first_of(delims, last);
    while (pos != std::string::npos || last != std::string::npos) {
        out.push_back(text.substr(last, pos - last));
        last = text.find_first_not_of(delims, pos);
        pos = text.find_first_of(delims, last);
    }
}

Circuit::Circuit() {
    const double s = 1.0 / std::sqrt(2.0);
    const double pi = 3.14159265358979323846;
    cplx h[4] = {s, s, s, -s};
    cplx x[4] = {0.0, 1.0, 1.0, 0.0};
    cplx z[4] = {1.0, 0.0, 0.0, -1.0};
    cplx y[4] = {0.0, cplx(0, 1), cplx(0, -1), 0.0};
    add_gate("H", h);
    add_gate("X", x);
    add_gate("Z", z);
    add_gate("Y", y);
    for (int k = 1; k <= 3; k++) {
        cplx r[4] = {1.0, 0.0, 0.0, std::polar(1.0, pi / double(1 << (k - 1)))};
        add_gate("R" + std::to_string(k), r);
    }
}

bool Circuit::add_gate(const std::string &name, const cplx m[4]) {
    if (gates.count(name)) return false;
    gates[name] = std::vector<cplx>(m, m + 4);
    return true;
}

namespace {
struct Group {
    std::vector<std::string> ops;
    std::vector<long> pos_ops;
    std::vector<long> ctrl;
    std::vector<long> pos_ctrl;
};
struct StepPT {
    int span;
    Op op;
};
}  // namespace

int Circuit::set_function(const std::string &function, int iterations, bool reset) {
    std::vector<std::string> steps;
    tokenize(function, steps, ";");
    if (reset) ops.clear();
    std::vector<Op> added;
    for (int it = 0; it < iterations; it++) {
        for (size_t si = 0; si < steps.size(); si++) {
            std::vector<std::string> toks;
            tokenize(steps[si], toks, ",");
            int nq = (int)toks.size();
            if (nq > 63) return fail(HGM_ERR_INVALID, "step %zu has %d qubits (max 63)", si, nq);
            std::map<long, Group> groups;
            for (int q = 0; q < nq; q++) {
                const std::string &tok = toks[q];
                size_t cpos = tok.find("Control"), tpos = tok.find("Target");
                size_t paren = tok.find("(") + 1;
                if (cpos != std::string::npos) {
                    long num = strtol(tok.c_str() + 7, nullptr, 10);
                    long val = strtol(tok.c_str() + paren, nullptr, 10);
                    groups[num].ctrl.push_back(val);
                    groups[num].pos_ctrl.push_back(q);
                } else if (tpos != std::string::npos) {
                    long num = strtol(tok.c_str() + 6, nullptr, 10);
                    if (paren == 0 || tok.size() < paren + 1)
                        return fail(HGM_ERR_INVALID, "malformed token '%s'", tok.c_str());
                    groups[num].ops.push_back(tok.substr(paren, tok.size() - paren - 1));
                    groups[num].pos_ops.push_back(q);
                } else if (tok != "ID") {
                    groups[0].ops.push_back(tok);
                    groups[0].pos_ops.push_back(q);
                }
            }
            std::vector<StepPT> step_pts;
            for (auto &kv : groups) {
                Group &g = kv.second;
                uint64_t cmask = 0, cval = 0;
                for (size_t c = 0; c < g.ctrl.size(); c++) {
                    int bit = nq - (int)g.pos_ctrl[c] - 1;
                    cmask += uint64_t(1) << bit;
                    if (g.ctrl[c]) cval += uint64_t(1) << bit;
                }
                for (size_t o = 0; o < g.ops.size(); o++) {
                    auto it2 = gates.find(g.ops[o]);
                    if (it2 == gates.end()) return fail(HGM_ERR_INVALID, "unknown gate '%s'", g.ops[o].c_str());
                    StepPT sp;
                    sp.span = nq - (int)g.pos_ops[o];
                    sp.op.target = sp.span - 1;
                    sp.op.cmask = cmask;
                    sp.op.cval = cval;
                    for (int k = 0; k < 4; k++) sp.op.m[k] = it2->second[k];
                    if (cmask & (uint64_t(1) << sp.op.target))
                        return fail(HGM_ERR_INVALID, "qubit %d is both control and target", (int)g.pos_ops[o]);
                    step_pts.push_back(sp);
                }
            }
            // odd steps: `increasing` = descending span; even: ascending.
            if (si % 2)
                std::sort(step_pts.begin(), step_pts.end(),
                          [](const StepPT &a, const StepPT &b) { return a.span > b.span; });
            else
                std::sort(step_pts.begin(), step_pts.end(),
                          [](const StepPT &a, const StepPT &b) { return a.span < b.span; });
            for (auto &sp : step_pts) added.push_back(sp.op);
            qubits = nq;
        }
    }
    ops.insert(ops.end(), added.begin(), added.end());
    pt_ptrs.clear();
    return HGM_OK;
}

}  // namespace hgm

using namespace hgm;

extern "C" {

const char *hgm_last_error(void) { return hgm::g_err; }

hgm_circuit *hgm_circuit_new(void) { return reinterpret_cast<hgm_circuit *>(new Circuit()); }

void hgm_circuit_free(hgm_circuit *c) { delete reinterpret_cast<Circuit *>(c); }

int hgm_circuit_add_gate(hgm_circuit *c, const char *name, const double m[8]) {
    if (!c || !name || !m) return -fail(HGM_ERR_INVALID, "null argument");
    cplx mm[4];
    for (int k = 0; k < 4; k++) mm[k] = cplx(m[2 * k], m[2 * k + 1]);
    return reinterpret_cast<Circuit *>(c)->add_gate(name, mm) ? 1 : 0;
}

int hgm_circuit_set_function(hgm_circuit *c, const char *steps, int iterations, int reset) {
    if (!c || !steps) return fail(HGM_ERR_INVALID, "null argument");
    if (iterations < 0) return fail(HGM_ERR_INVALID, "negative iterations");
    return reinterpret_cast<Circuit *>(c)->set_function(steps, iterations, reset != 0);
}

int hgm_circuit_append_op(hgm_circuit *c, int target, int64_t cmask, int64_t cval, const double m[8]) {
    if (!c || !m) return fail(HGM_ERR_INVALID, "null argument");
    if (target < 0 || target > 62) return fail(HGM_ERR_INVALID, "target %d out of range", target);
    if ((uint64_t)cmask & (uint64_t(1) << target)) return fail(HGM_ERR_INVALID, "target is also a control");
    if (((uint64_t)cval & ~(uint64_t)cmask) != 0) return fail(HGM_ERR_INVALID, "control value outside mask");
    Circuit *cc = reinterpret_cast<Circuit *>(c);
    Op op;
    op.target = target;
    op.cmask = (uint64_t)cmask;
    op.cval = (uint64_t)cval;
    for (int k = 0; k < 4; k++) op.m[k] = cplx(m[2 * k], m[2 * k + 1]);
    cc->ops.push_back(op);
    cc->pt_ptrs.clear();
    return HGM_OK;
}

int hgm_circuit_qubits(const hgm_circuit *c) { return c ? reinterpret_cast<const Circuit *>(c)->qubits : 0; }

int64_t hgm_circuit_num_ops(const hgm_circuit *c) {
    return c ? (int64_t) reinterpret_cast<const Circuit *>(c)->ops.size() : 0;
}

int hgm_circuit_get_ops(const hgm_circuit *c, int32_t *target, int64_t *cmask, int64_t *cval, double *m) {
    if (!c) return fail(HGM_ERR_INVALID, "null circuit");
    const Circuit *cc = reinterpret_cast<const Circuit *>(c);
    for (size_t i = 0; i < cc->ops.size(); i++) {
        const Op &op = cc->ops[i];
        if (target) target[i] = op.target;
        if (cmask) cmask[i] = (int64_t)op.cmask;
        if (cval) cval[i] = (int64_t)op.cval;
        if (m)
            for (int k = 0; k < 4; k++) {
                m[8 * i + 2 * k] = op.m[k].real();
                m[8 * i + 2 * k + 1] = op.m[k].imag();
            }
    }
    return HGM_OK;
}

void *hgm_circuit_ref_pts(hgm_circuit *c, int precision) {
    if (!c) {
        fail(HGM_ERR_INVALID, "null circuit");
        return nullptr;
    }
    Circuit *cc = reinterpret_cast<Circuit *>(c);
    size_t n = cc->ops.size();
    size_t amp = precision == HGM_F64 ? 16 : 8;
    cc->pt_storage.assign(n * sizeof(RefPTLayout), 0);
    cc->mat_storage.assign(n * 4 * amp, 0);
    cc->pt_ptrs.assign(n + 1, nullptr);
    for (size_t i = 0; i < n; i++) {
        const Op &op = cc->ops[i];
        RefPTLayout *pt = reinterpret_cast<RefPTLayout *>(&cc->pt_storage[i * sizeof(RefPTLayout)]);
        unsigned char *mat = &cc->mat_storage[i * 4 * amp];
        for (int k = 0; k < 4; k++) {
            if (precision == HGM_F64) {
                double v[2] = {op.m[k].real(), op.m[k].imag()};
                memcpy(mat + k * 16, v, 16);
            } else {
                float v[2] = {(float)op.m[k].real(), (float)op.m[k].imag()};
                memcpy(mat + k * 8, v, 8);
            }
        }
        pt->qubits = 1;
        pt->matrix = mat;
        pt->matrix_size = 2;
        pt->span_start_bit = op.target + 1;
        pt->target_bit = op.target;
        pt->affected = false;
        pt->control_value = (long)op.cval;
        pt->control_mask = (long)op.cmask;
        pt->control_count = __builtin_popcountll(op.cmask);
        cc->pt_ptrs[i] = pt;
    }
    cc->pt_ptrs[n] = nullptr;
    return cc->pt_ptrs.data();
}

}  // extern "C"
