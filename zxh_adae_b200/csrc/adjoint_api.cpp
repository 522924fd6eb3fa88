// adjoint_api.cpp -- zxh_expectation, zxh_adjoint_gradient and zxh_gate_count.
//
// No counterpart in the reference: ZXH-Sim has no observables or gradients. The
// sweep reuses the execute() walk and planner for the forward pass and works in
// the real-address space of the affine map throughout.
//
// Forward: the recorded gates run with every qubit expanded from the start
// (eager_expand_all, zxh.cpp:721-729) and X/CX transported through the map, in
// segments that end after every `checkpoint_every` parameterised gates; the state
// after each segment is copied aside. With all qubits expanded the map never
// gains a column, so undoing X/CX on the map while walking the gates backwards
// gives back, at every gate boundary, exactly the map the forward pass had there,
// and a checkpoint is a plain copy into the reverse state.
//
// Reverse: psi (a copy of the forward output) and lambda = H psi walk back over
// the gates. A 2x2 gate is one adj_pair pass that reduces its gradient and
// uncomputes both states with U^dagger; a run of diagonal gates (RZ, P, CP, Z,
// with X/CX relabelings between them) is one adj_diag pass that reduces every
// gradient of the run at once, which is exact because the run's gates commute.
//
// Global phase: Z/RZ records carry a global phase that the walk keeps outside the
// state (zxh.cpp:477-493). psi and lambda carry the same untracked factor, so
// Im<lambda|G|psi> does not see it, and a checkpoint's factor differs from the
// reverse state's only by rounding of the accumulated phase.
#include "adjoint.h"
#include "adjoint_host.h"
#include "sim.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

using namespace zxh::api;

namespace zxh {
namespace adj {

// gradient generator of a lowered 2x2 record: RY = U3(theta, 0, 0), RX =
// U3(theta, pi/2, -pi/2) (the lowering of zxh_rx and ZXH_GATE_RX)
uint32_t pair_generator(const Gate &g)
{
    if (g.type != zxh::G_U3) return 0;
    if (g.lambda == 0.0 && g.phi == 0.0) return 1;
    if (g.lambda == kPi / 2.0 && g.phi == -kPi / 2.0) return 2;
    return 0;
}

bool parameterised(const Gate &g)
{
    switch (g.type) {
    case zxh::G_RZ:
    case zxh::G_P:
    case zxh::G_CP: return true;
    case zxh::G_U3: return pair_generator(g) != 0;
    default: return false;
    }
}

// Terms in the real-address form of map A over m bits. X terms on a qubit whose
// flip leaves the map's image are dropped when drop_unreachable is set (their
// expectation is exactly zero) and rejected otherwise.
int compile_terms(zxh_sim *s, const zxh_term *terms, size_t nterms, AffineMap &A, int m, bool drop_unreachable,
                  std::vector<TermDev> &out)
{
    out.clear();
    if (nterms && !terms) return fail(s, ZXH_ERR_ARG, "terms is null");
    if (nterms > zxh::kMaxTerms)
        return fail(s, ZXH_ERR_LIMIT, "at most " + std::to_string(zxh::kMaxTerms) + " observable terms");
    for (size_t i = 0; i < nterms; i++) {
        const zxh_term &t = terms[i];
        TermDev d;
        std::memset(&d, 0, sizeof(d));
        d.kind = t.kind;
        d.coef = t.coef;
        if (t.q0 >= s->n || (t.kind == ZXH_TERM_ZZ && t.q1 >= s->n))
            return fail(s, ZXH_ERR_ARG, "observable term qubit out of range");
        switch (t.kind) {
        case ZXH_TERM_ZZ: {
            const zxh::Sel s1 = A.selector(int(t.q1));
            d.a1 = s1.alpha;
            d.b1 = uint32_t(s1.beta);
        }
            // fall through
        case ZXH_TERM_Z: {
            const zxh::Sel s0 = A.selector(int(t.q0));
            d.a0 = s0.alpha;
            d.b0 = uint32_t(s0.beta);
            break;
        }
        case ZXH_TERM_X: {
            uint64_t delta = 0;
            if (!A.solve(int(t.q0), delta)) {
                if (drop_unreachable) continue;
                return fail(s, ZXH_ERR_STATE, "X term on a qubit the state does not span");
            }
            d.delta = delta & zxh::low_mask(m);
            break;
        }
        default: return fail(s, ZXH_ERR_ARG, "unknown observable term kind " + std::to_string(t.kind));
        }
        out.push_back(d);
    }
    // X terms first: the lambda kernels issue their gathers back to back
    std::stable_partition(out.begin(), out.end(), [](const TermDev &t) { return t.kind == ZXH_TERM_X; });
    return ZXH_OK;
}

// Region layout of d_adj: grads | energy | terms | exp table | grow-pass blob.
struct AdjLayout {
    size_t grads, energy, terms, exp, grow, total;
    AdjLayout(size_t ngrads, size_t nterms, size_t grow_bytes = 0)
    {
        auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
        grads = 0;
        energy = up(ngrads * sizeof(double));
        terms = energy + 256;
        exp = up(terms + nterms * sizeof(TermDev));
        grow = up(exp + (size_t(16) << zxh::kExpTableBits));
        total = grow + up(grow_bytes);
    }
};

// Descriptors of the general strided adjoint passes, packed into one blob.
std::vector<uint8_t> pack_grow(std::vector<RevStep> &steps)
{
    std::vector<uint8_t> blob;
    auto put = [&](const void *p, size_t n) -> uint64_t {
        const uint64_t off = (blob.size() + 15) & ~uint64_t(15);
        blob.resize(off + n + 16, 0);
        if (n) std::memcpy(blob.data() + off, p, n);
        return off;
    };
    uint64_t toff = 0;
    bool have_tab = false;
    for (RevStep &r : steps) {
        if (r.kind != RevStep::GROW) continue;
        zxh::GrowBuild &gb = r.gb;
        if (gb.dev.ncls[1][2] && !have_tab) {  // the phase table of the windows
            std::vector<uint8_t> t;
            zxh::exp_table(gb.elem_bytes, t);
            toff = put(t.data(), t.size());
            have_tab = true;
        }
        r.toff = toff;
        gb.dev.nsel = uint32_t(gb.sels.size());
        gb.dev.off_gates = put(gb.gates.data(), gb.gates.size() * sizeof(zxh::GrowGateDev));
        gb.dev.off_sel = put(gb.sels.data(), gb.sels.size() * sizeof(zxh::GrowSelDev));
        gb.dev.off_terms[0] = put(gb.terms[0].data(), gb.terms[0].size() * sizeof(zxh::GrowTermDev));
        gb.dev.off_terms[1] = put(gb.terms[1].data(), gb.terms[1].size() * sizeof(zxh::GrowTermDev));
        r.off = put(&gb.dev, sizeof(zxh::GrowDev));
    }
    return blob;
}

// Forward pass in segments [0, ends[0]), [ends[0], ends[1]), ... with every qubit
// expanded; the state after segment k < ends.size() - 1 is saved as checkpoint k.
// wait = false: returns once everything is queued (the caller waits, reads the
// status word, which stays set for it, and the time between evf0 and evf1).
int forward_segments(zxh_sim *s, const std::vector<size_t> &ends, double &ms, uint64_t &kernels, bool wait = true)
{
    const int N = int(s->n);
    const size_t bytes = size_t(s->elem_bytes) << N;
    if (int rc = ensure_dev(s, &s->d_state, s->state_cap_bytes, std::max<size_t>(bytes, 256), "cudaMalloc(state)"))
        return rc;
    const size_t nck = ends.empty() ? 0 : ends.size() - 1;
    if (nck)
        if (int rc = ensure_dev(s, &s->d_ckpt, s->ckpt_cap, nck * bytes, "cudaMalloc(checkpoints)")) return rc;
    s->M = N;
    s->executed = false;
    s->measured = 0;
    zxh::WalkState &ws = s->ws;
    ws.map.reset(N);
    for (int q = 0; q < N; q++) ws.map.append_col(q);
    ws.m = N;
    ws.gphase = zxh::cd(1.0, 0.0);
    ws.fresh = true;
    ws.init_bits = N;
    ms = 0.0;
    kernels = 0;
    // every segment is planned on the host first, its program uploaded in one
    // copy, then all passes and checkpoint saves are queued and waited for once
    std::vector<zxh::Plan> plans(ends.size());
    std::vector<size_t> boff(ends.size());
    size_t total = 0, a = 0;
    for (size_t k = 0; k < ends.size(); k++) {
        const zxh::WalkState start = ws;
        std::vector<zxh::Op> ops;
        std::string err;
        if (int rc = zxh::walk(s->gates.data() + a, ends[k] - a, false, N, ws, ops, err)) return fail(s, rc, err);
        if (int rc = zxh::plan(ops, s->elem_bytes, s->pp, start, plans[k], err)) return fail(s, rc, err);
        ws.fresh = false;
        boff[k] = total;
        total += (plans[k].blob.size() + 255) & ~size_t(255);
        a = ends[k];
    }
    total = std::max<size_t>(total, 256);
    if (total > s->stage_cap) {
        if (s->h_stage) cudaFreeHost(s->h_stage);
        s->h_stage = nullptr;
        s->stage_cap = 0;
        CK(s, cudaMallocHost(reinterpret_cast<void **>(&s->h_stage), total * 2), "cudaMallocHost(program)");
        s->stage_cap = total * 2;
    }
    if (int rc = ensure_dev(s, reinterpret_cast<void **>(&s->d_blob), s->blob_cap, s->stage_cap, "cudaMalloc(program)"))
        return rc;
    for (size_t k = 0; k < ends.size(); k++) std::memcpy(s->h_stage + boff[k], plans[k].blob.data(), plans[k].blob.size());
    CK(s, cudaMemcpyAsync(s->d_blob, s->h_stage, total, cudaMemcpyHostToDevice, s->stream), "upload programs");
    if (!s->evf0) CK(s, cudaEventCreate(&s->evf0), "event");
    if (!s->evf1) CK(s, cudaEventCreate(&s->evf1), "event");
    CK(s, cudaMemsetAsync(s->d_status, 0, sizeof(zxh::DevStatus), s->stream), "reset status");
    CK(s, cudaEventRecord(s->evf0, s->stream), "event");
    // cur: where the state after the segments so far lives (the state buffer or a
    // checkpoint slot); a general strided pass at a segment's end writes straight
    // into the slot and the next segment's first one reads from it
    auto ckpt = [&](size_t k) { return static_cast<void *>(static_cast<uint8_t *>(s->d_ckpt) + k * bytes); };
    void *cur = s->d_state;
    auto to_state = [&]() -> int {
        if (cur != s->d_state)
            CK(s, cudaMemcpyAsync(s->d_state, cur, bytes, cudaMemcpyDeviceToDevice, s->stream), "load checkpoint");
        cur = s->d_state;
        return ZXH_OK;
    };
    for (size_t k = 0; k < ends.size(); k++) {
        const std::vector<zxh::Pass> &P = plans[k].passes;
        if (!P.empty()) {
            const void *src = nullptr;
            if (cur != s->d_state) {
                if (P.front().kind == zxh::Pass::GROW) src = cur;
                else if (int rc = to_state()) return rc;
            }
            void *dst = (k < nck && P.back().kind == zxh::Pass::GROW) ? ckpt(k) : nullptr;
            if (dst == src && dst) dst = nullptr;  // never in place on a slot it reads whole
            CK(s, zxh::run_passes(P, s->d_blob + boff[k], s->d_state, s->elem_bytes, s->d_status, s->sms, s->stream,
                                  kernels, src, dst),
               "launch");
            cur = dst ? dst : s->d_state;
        }
        if (k < nck && cur != ckpt(k))
            CK(s, cudaMemcpyAsync(ckpt(k), cur, bytes, cudaMemcpyDeviceToDevice, s->stream), "save checkpoint");
    }
    if (int rc = to_state()) return rc;  // the forward output stays in the state buffer
    CK(s, cudaEventRecord(s->evf1, s->stream), "event");
    if (!wait) {
        s->executed = true;
        return ZXH_OK;
    }
    CK(s, cudaMemcpyAsync(s->h_status, s->d_status, sizeof(zxh::DevStatus), cudaMemcpyDeviceToHost, s->stream),
       "read status");
    CK(s, cudaStreamSynchronize(s->stream), "forward");
    float fms = 0.0f;
    CK(s, cudaEventElapsedTime(&fms, s->evf0, s->evf1), "event time");
    ms = double(fms);
    if (s->h_status->code != 0)
        return fail(s, int(s->h_status->code), "device wait gave up (site " + std::to_string(s->h_status->where) + ")");
    s->executed = true;
    return ZXH_OK;
}

// The reverse program: gates walked backwards from the forward output's map.
int reverse_program(zxh_sim *s, const std::vector<size_t> &ends, AffineMap A, std::vector<RevStep> &steps,
                    std::vector<AdjDiagGate> &dgates, std::vector<uint32_t> &dslots, int diag_max)
{
    const int N = int(s->n);
    const size_t count = s->gates.size();
    long open = -1;                    // diagonal group being filled (states too small for strided passes)
    size_t next_ck = ends.size() - 1;  // checkpoints are restored from the last one down
    const int F = zxh::grow_fixed_bits(s->elem_bytes);
    const int R = std::max(1, std::min(s->pp.adj_regs, zxh::grow_reg_bits(s->elem_bytes, true)));
    const int maxg = zxh::grow_adjoint_gates();
    const bool fuse = N >= F && s->pp.adj_windows;  // diagonal gates ride in the general strided passes
    PairGroup pg;
    // Diagonal gates met since the last pair group: in forward order they follow the
    // gates of the group collected next, so that group's pass undoes them first.
    std::vector<zxh::DiagTerm> pw;
    std::vector<uint32_t> pwk, pws;
    auto pair_steps = [&]() {  // one global pair pass per gate
        for (const PairGroup::G &g : pg.gates) {
            RevStep p;
            p.kind = RevStep::PAIR;
            std::memset(&p.pair, 0, sizeof(p.pair));
            p.pair.m = uint32_t(N);
            p.pair.pivot = uint32_t(__builtin_ctzll(g.op.delta));
            p.pair.delta = g.op.delta;
            p.pair.alpha = g.op.sel.alpha;
            p.pair.beta = uint32_t(g.op.sel.beta);
            p.pair.gen = g.gen;
            for (int k = 0; k < 4; k++) {
                p.pair.u[2 * k] = g.op.u[k].real();
                p.pair.u[2 * k + 1] = g.op.u[k].imag();
            }
            p.slot = g.slot;
            steps.push_back(p);
        }
    };
    auto window_steps = [&]() -> bool {  // the pending window alone, in chunks that fit
        for (size_t a = 0; a < pw.size(); a += 32) {
            const size_t e = std::min(pw.size(), a + 32);
            const std::vector<zxh::DiagTerm> w(pw.begin() + long(a), pw.begin() + long(e));
            const std::vector<uint32_t> k(pwk.begin() + long(a), pwk.begin() + long(e));
            const std::vector<uint32_t> sl(pws.begin() + long(a), pws.begin() + long(e));
            RevStep r;
            r.kind = RevStep::GROW;
            if (!r.gb.init(s->elem_bytes, N, std::vector<uint64_t>()) || !r.gb.add_window(1, w, &k, &sl, true))
                return false;
            steps.push_back(r);
        }
        return true;
    };
    auto close_group = [&]() -> int {
        if (pg.gates.empty() && pw.empty()) return ZXH_OK;
        std::vector<uint64_t> regs;
        for (const PairGroup::G &g : pg.gates)
            if (g.op.delta >> F) regs.push_back(g.op.delta);
        RevStep r;
        r.kind = RevStep::GROW;
        bool ok = fuse && r.gb.init(s->elem_bytes, N, regs);
        for (const PairGroup::G &g : pg.gates) ok = ok && r.gb.add_gate(g.op, g.gen, g.slot, true);
        if (ok && (pw.empty() || r.gb.add_window(1, pw, &pwk, &pws, true))) {
            steps.push_back(r);
        } else {
            if (!pw.empty() && !window_steps()) return fail(s, ZXH_ERR_STATE, "adjoint sweep: window not placeable");
            if (!pg.gates.empty()) {
                RevStep r2;
                r2.kind = RevStep::GROW;
                bool ok2 = fuse && r2.gb.init(s->elem_bytes, N, regs);
                for (const PairGroup::G &g : pg.gates) ok2 = ok2 && r2.gb.add_gate(g.op, g.gen, g.slot, true);
                if (ok2) steps.push_back(r2);
                else pair_steps();
            }
        }
        pg = PairGroup();
        pw.clear();
        pwk.clear();
        pws.clear();
        return ZXH_OK;
    };
    for (size_t gi = count; gi-- > 0;) {
        if (next_ck > 0 && ends[next_ck - 1] == gi + 1) {
            if (int rc = close_group()) return rc;
            next_ck--;
            RevStep r;
            r.kind = RevStep::RESTORE;
            r.ckpt = next_ck;
            steps.push_back(r);
            open = -1;
        }
        const Gate &g = s->gates[gi];
        switch (g.type) {
        case zxh::G_X: A.flip_b(int(g.q)); break;
        case zxh::G_CX:
            if (int rc = close_group()) return rc;
            A.row_xor(int(g.q), int(g.cq));
            A.b_xor(int(g.q), int(g.cq));
            break;
        case zxh::G_Z:
        case zxh::G_RZ:
        case zxh::G_P:
        case zxh::G_CP: {
            const uint32_t kind = g.type == zxh::G_Z ? 0 : g.type == zxh::G_RZ ? 1 : 2;
            const double th = g.type == zxh::G_Z ? kPi : g.theta;
            const zxh::Sel s0 = A.selector(int(g.type == zxh::G_CP ? g.cq : g.q));
            const zxh::Sel s1 = A.selector(int(g.q));
            if (fuse) {
                if (!pg.gates.empty() || pw.size() >= size_t(zxh::kGrowMaxTerms))
                    if (int rc = close_group()) return rc;
                zxh::DiagTerm t;
                t.s0 = s0;
                t.s1 = s1;
                t.two = g.type == zxh::G_CP;
                t.theta = th;
                pw.push_back(t);
                pwk.push_back(kind);
                pws.push_back(uint32_t(gi));
                break;
            }
            if (open < 0 || steps[size_t(open)].ng == uint32_t(diag_max)) {
                RevStep r;
                r.kind = RevStep::DIAG;
                r.first = dgates.size();
                steps.push_back(r);
                open = long(steps.size()) - 1;
            }
            AdjDiagGate d;
            std::memset(&d, 0, sizeof(d));
            d.a0 = s0.alpha;
            d.b0 = uint32_t(s0.beta);
            if (g.type == zxh::G_CP) {
                d.a1 = s1.alpha;
                d.b1 = uint32_t(s1.beta);
                d.two = 1;
            }
            d.kind = kind;
            d.tq = zxh::phase_turns(th);
            d.m0 = kind == 1 ? 1.0 : 0.0;
            d.m1 = kind == 1 ? -1.0 : kind == 2 ? -2.0 : 0.0;
            dgates.push_back(d);
            dslots.push_back(uint32_t(gi));
            steps[size_t(open)].ng++;
            break;
        }
        case zxh::G_H:
        case zxh::G_U3: {
            open = -1;
            PairGroup::G pgt;
            uint64_t delta = 0;
            if (!A.solve(int(g.q), delta)) return fail(s, ZXH_ERR_STATE, "adjoint sweep: qubit outside the map");
            pgt.op.delta = delta & zxh::low_mask(N);
            pgt.op.sel = A.selector(int(g.q));
            if (g.type == zxh::G_H) zxh::u3_matrix(kPi / 2.0, kPi, 0.0, pgt.op.u);
            else zxh::u3_matrix(g.theta, g.lambda, g.phi, pgt.op.u);
            pgt.gen = pair_generator(g);
            pgt.slot = uint32_t(gi);
            pgt.q = int(g.q);
            if (!pg.fits(pgt, F, R, N, maxg))
                if (int rc = close_group()) return rc;
            pg.add(pgt, F);
            break;
        }
        default: break;
        }
    }
    return close_group();
}

}  // namespace adj
}  // namespace zxh

using namespace zxh::adj;
using zxh::AdjDiagGate;
using zxh::AffineMap;
using zxh::TermDev;

extern "C" {

int zxh_gate_count(const zxh_sim *s, size_t *out)
{
    if (!s || !out) return ZXH_ERR_ARG;
    *out = s->gates.size();
    return ZXH_OK;
}

int zxh_expectation(zxh_sim *s, const zxh_term *terms, size_t nterms, double *value)
{
    if (!s) return ZXH_ERR_ARG;
    if (!value) return fail(s, ZXH_ERR_ARG, "value is null");
    if (!s->executed) return fail(s, ZXH_ERR_STATE, "expectation requires execute() first");
    if (int rc = use_device(s)) return rc;
    if (int rc = flush_pending(s)) return rc;
    std::vector<TermDev> dt;
    if (int rc = compile_terms(s, terms, nterms, s->ws.map, s->ws.m, true, dt)) return rc;
    const AdjLayout L(0, dt.size());
    if (int rc = ensure_dev(s, reinterpret_cast<void **>(&s->d_adj), s->adj_cap, L.total, "cudaMalloc(adjoint)"))
        return rc;
    double *d_energy = reinterpret_cast<double *>(s->d_adj + L.energy);
    auto *d_terms = reinterpret_cast<TermDev *>(s->d_adj + L.terms);
    CK(s, cudaMemsetAsync(d_energy, 0, sizeof(double), s->stream), "reset energy");
    if (!dt.empty())
        CK(s, cudaMemcpyAsync(d_terms, dt.data(), dt.size() * sizeof(TermDev), cudaMemcpyHostToDevice, s->stream),
           "upload terms");
    CK(s, cudaEventRecord(s->ev0, s->stream), "event");
    CK(s, zxh::run_lambda(s->d_state, nullptr, s->ws.m, s->elem_bytes, d_terms, uint32_t(dt.size()), d_energy, s->sms,
                          s->stream),
       "expectation launch");
    CK(s, cudaEventRecord(s->ev1, s->stream), "event");
    CK(s, cudaMemcpyAsync(value, d_energy, sizeof(double), cudaMemcpyDeviceToHost, s->stream), "read energy");
    CK(s, cudaStreamSynchronize(s->stream), "expectation");
    CK(s, cudaEventElapsedTime(&s->last_ms, s->ev0, s->ev1), "event time");
    s->stat_kernels = 1;
    s->stat_passes = 1;
    return ZXH_OK;
}

int zxh_adjoint_gradient(zxh_sim *s, const zxh_term *terms, size_t nterms, size_t checkpoint_every, double *value,
                         double *grads, size_t ngrads)
{
    if (!s) return ZXH_ERR_ARG;
    const size_t count = s->gates.size();
    if (!value) return fail(s, ZXH_ERR_ARG, "value is null");
    if (count && !grads) return fail(s, ZXH_ERR_ARG, "grads is null");
    if (ngrads < count) return fail(s, ZXH_ERR_ARG, "grads holds fewer entries than recorded gates");
    if (s->n > 40) return fail(s, ZXH_ERR_LIMIT, "the adjoint sweep holds 2^n amplitudes: n must be at most 40");
    for (size_t i = 0; i < nterms && terms; i++)
        if (terms[i].kind < ZXH_TERM_Z || terms[i].kind > ZXH_TERM_X)
            return fail(s, ZXH_ERR_ARG, "unknown observable term kind " + std::to_string(terms[i].kind));
    if (nterms > zxh::kMaxTerms)
        return fail(s, ZXH_ERR_LIMIT, "at most " + std::to_string(zxh::kMaxTerms) + " observable terms");
    if (int rc = use_device(s)) return rc;
    s->pending.clear();  // the forward segments rebuild the state from |0...0>
    const int N = int(s->n);

    // forward segments
    std::vector<size_t> ends;
    size_t np = 0;
    for (size_t i = 0; i < count; i++)
        if (parameterised(s->gates[i]) && checkpoint_every && ++np % checkpoint_every == 0 && i + 1 < count)
            ends.push_back(i + 1);
    ends.push_back(count);
    double fwd_ms = 0.0;
    uint64_t kernels = 0;
    // queued, not waited for: the reverse program is planned on the host while
    // the forward passes run. Every return from here on waits for the stream
    // first, so an early error never leaves queued work reading the pinned
    // program buffer that the next call refills.
    struct WaitOnExit {
        zxh_sim *s;
        ~WaitOnExit() { cudaStreamSynchronize(s->stream); }
    } wait_on_exit{s};
    if (int rc = forward_segments(s, ends, fwd_ms, kernels, false)) return rc;

    // reverse program
    AffineMap A = s->ws.map;
    std::vector<TermDev> dt;
    if (int rc = compile_terms(s, terms, nterms, A, N, false, dt)) return rc;
    std::vector<RevStep> steps;
    std::vector<AdjDiagGate> dgates;
    std::vector<uint32_t> dslots;
    if (int rc = reverse_program(s, ends, A, steps, dgates, dslots)) return rc;

    // device buffers
    const size_t bytes = size_t(s->elem_bytes) << N;
    if (int rc = ensure_dev(s, &s->d_psi, s->psi_cap, bytes, "cudaMalloc(adjoint psi)")) return rc;
    if (int rc = ensure_dev(s, &s->d_lam, s->lam_cap, bytes, "cudaMalloc(adjoint lambda)")) return rc;
    const std::vector<uint8_t> gblob = pack_grow(steps);
    const AdjLayout L(count, dt.size(), gblob.size());
    if (int rc = ensure_dev(s, reinterpret_cast<void **>(&s->d_adj), s->adj_cap, L.total, "cudaMalloc(adjoint)"))
        return rc;
    if (!gblob.empty())
        CK(s, cudaMemcpyAsync(s->d_adj + L.grow, gblob.data(), gblob.size(), cudaMemcpyHostToDevice, s->stream),
           "upload pass descriptors");
    double *d_grads = reinterpret_cast<double *>(s->d_adj + L.grads);
    double *d_energy = reinterpret_cast<double *>(s->d_adj + L.energy);
    auto *d_terms = reinterpret_cast<TermDev *>(s->d_adj + L.terms);
    CK(s, cudaMemsetAsync(s->d_adj, 0, L.terms, s->stream), "reset gradients");
    if (!dt.empty())
        CK(s, cudaMemcpyAsync(d_terms, dt.data(), dt.size() * sizeof(TermDev), cudaMemcpyHostToDevice, s->stream),
           "upload terms");
    std::vector<uint8_t> etab;
    if (!dgates.empty()) {
        zxh::exp_table(s->elem_bytes, etab);
        CK(s, cudaMemcpyAsync(s->d_adj + L.exp, etab.data(), etab.size(), cudaMemcpyHostToDevice, s->stream),
           "upload phase table");
    }

    // reverse sweep (the status word was reset before the forward passes and
    // keeps a forward failure)
    CK(s, cudaEventRecord(s->ev0, s->stream), "event");
    CK(s, cudaMemcpyAsync(s->d_psi, s->d_state, bytes, cudaMemcpyDeviceToDevice, s->stream), "copy state");
    CK(s, zxh::run_lambda(s->d_psi, s->d_lam, N, s->elem_bytes, d_terms, uint32_t(dt.size()), d_energy, s->sms,
                          s->stream),
       "lambda launch");
    kernels++;
    // A checkpoint is not copied back into psi: the next general strided pass
    // reads psi from it (and writes psi); any other kernel gets the copy first.
    const void *psi_from = nullptr;
    auto settle_restore = [&]() -> int {
        if (psi_from) {
            CK(s, cudaMemcpyAsync(s->d_psi, psi_from, bytes, cudaMemcpyDeviceToDevice, s->stream),
               "restore checkpoint");
            psi_from = nullptr;
        }
        return ZXH_OK;
    };
    for (const RevStep &r : steps) {
        if (r.kind != RevStep::GROW && r.kind != RevStep::RESTORE)
            if (int rc = settle_restore()) return rc;
        switch (r.kind) {
        case RevStep::RESTORE:
            if (int rc = settle_restore()) return rc;
            psi_from = static_cast<uint8_t *>(s->d_ckpt) + r.ckpt * bytes;
            break;
        case RevStep::PAIR:
            CK(s, zxh::run_adj_pair(s->d_psi, s->d_lam, s->elem_bytes, r.pair, d_grads + r.slot, s->sms, s->stream),
               "adjoint pair launch");
            kernels++;
            break;
        case RevStep::GROW:
            CK(s, zxh::run_grow(s->d_adj + L.grow, r.off, r.toff, int(r.gb.regs.size()), r.gb.dev.nitems, s->elem_bytes,
                                s->d_psi, s->d_lam, d_grads, r.gb.all_real(),
                                (s->pp.grow_staged & (s->elem_bytes == 8 ? 1 : 4)) != 0,
                                s->d_status, s->sms, s->stream, psi_from),
               "adjoint strided launch");
            psi_from = nullptr;
            kernels++;
            break;
        case RevStep::DIAG:
            CK(s, zxh::run_adj_diag(s->d_psi, s->d_lam, N, s->elem_bytes, dgates.data() + r.first, r.ng, d_grads,
                                    dslots.data() + r.first, s->d_adj + L.exp, s->sms, s->stream),
               "adjoint diagonal launch");
            kernels++;
            break;
        }
    }
    if (int rc = settle_restore()) return rc;  // psi ends as the sweep's last state
    CK(s, cudaEventRecord(s->ev1, s->stream), "event");
    CK(s, cudaMemcpyAsync(s->h_status, s->d_status, sizeof(zxh::DevStatus), cudaMemcpyDeviceToHost, s->stream),
       "read status");
    CK(s, cudaMemcpyAsync(value, d_energy, sizeof(double), cudaMemcpyDeviceToHost, s->stream), "read energy");
    if (count)
        CK(s, cudaMemcpyAsync(grads, d_grads, count * sizeof(double), cudaMemcpyDeviceToHost, s->stream),
           "read gradients");
    CK(s, cudaStreamSynchronize(s->stream), "adjoint sweep");
    if (s->h_status->code != 0)
        return fail(s, int(s->h_status->code),
                    "device wait gave up (site " + std::to_string(s->h_status->where) + ")");
    float rev_ms = 0.0f, f_ms = 0.0f;
    CK(s, cudaEventElapsedTime(&rev_ms, s->ev0, s->ev1), "event time");
    CK(s, cudaEventElapsedTime(&f_ms, s->evf0, s->evf1), "event time");
    fwd_ms = double(f_ms);
    s->last_ms = float(fwd_ms + double(rev_ms));
    s->stat_kernels = kernels;
    s->stat_passes = steps.size() + 1;
    return ZXH_OK;
}

}  // extern "C"
