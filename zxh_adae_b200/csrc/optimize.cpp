// optimize.cpp -- the host circuit compiler: the reference's boundary scheduler
// (src/zxh/zxhsim/circ_optimizer.py:218-420) over this library's gate records.
//
// Single-qubit gates accumulate per qubit as one pending 2x2 matrix (up to a
// global phase) until a two-qubit gate or a barrier needs the qubit. A flushed
// matrix is classified as the reference does (_classify_pending, :97-126):
// identity (nothing), X^x P(theta) (an RZ and maybe an X: diagonal and map-only
// work in the simulator), P(near) H P(far) (an H when it is exactly H, else a
// U3), or general (a U3). At a CX whose two qubits both hold exactly H, the CX is
// emitted reversed and the H's stay pending (H (x) H . CX(c, t) = CX(t, c) .
// H (x) H, :318-327): H gates that would expand the state cancel across CX
// chains, which lowers the required state bits M and the pass count. Results
// equal the input circuit up to a global phase.
#include "../../include/zxh_b200.h"
#include "host.h"
#include "sim.h"

#include <cmath>
#include <complex>
#include <string>
#include <vector>

namespace {

using cd = std::complex<double>;
constexpr double kPi = 3.14159265358979323846;
constexpr double kAtol = 1e-9;  // _ATOL (circ_optimizer.py:14)
constexpr double kRtol = 1e-5;  // numpy.allclose's relative tolerance, which the reference's checks inherit

struct M2 {
    cd a[4];  // row major: m00, m01, m10, m11
};

M2 mul(const M2 &x, const M2 &y)
{
    M2 r;
    r.a[0] = x.a[0] * y.a[0] + x.a[1] * y.a[2];
    r.a[1] = x.a[0] * y.a[1] + x.a[1] * y.a[3];
    r.a[2] = x.a[2] * y.a[0] + x.a[3] * y.a[2];
    r.a[3] = x.a[2] * y.a[1] + x.a[3] * y.a[3];
    return r;
}

M2 ident() { return M2{{1.0, 0.0, 0.0, 1.0}}; }
M2 had()
{
    const double h = 1.0 / std::sqrt(2.0);
    return M2{{h, h, h, -h}};
}
M2 pauli_x() { return M2{{0.0, 1.0, 1.0, 0.0}}; }

double norm_angle(double t) { return std::atan2(std::sin(t), std::cos(t)); }

M2 phase_m(double t) { return M2{{1.0, 0.0, 0.0, std::polar(1.0, norm_angle(t))}}; }

bool close(cd a, cd b, double atol) { return std::abs(a - b) <= atol + kRtol * std::abs(b); }

// lhs == e^{i g} rhs for some g (_matrix_equiv_up_to_phase, :45-66)
bool equiv_up_to_phase(const M2 &l, const M2 &r)
{
    cd scale = 0.0;
    bool have = false;
    for (int k = 0; k < 4 && !have; k++) {
        if (std::abs(r.a[k]) > kAtol) {
            if (std::abs(l.a[k]) <= kAtol) return false;
            scale = l.a[k] / r.a[k];
            have = true;
        } else if (std::abs(l.a[k]) > kAtol) {
            return false;
        }
    }
    if (!have) {
        for (int k = 0; k < 4; k++)
            if (!close(l.a[k], r.a[k], kAtol)) return false;
        return true;
    }
    if (std::abs(scale) <= kAtol) return false;
    scale /= std::abs(scale);
    for (int k = 0; k < 4; k++)
        if (!close(l.a[k], scale * r.a[k], kAtol)) return false;
    return true;
}

// divides by the phase of the first entry above the tolerance (:37-42)
M2 drop_phase(const M2 &m)
{
    M2 o = m;
    for (int k = 0; k < 4; k++)
        if (std::abs(m.a[k]) > kAtol) {
            const cd ph = m.a[k] / std::abs(m.a[k]);
            for (int j = 0; j < 4; j++) o.a[j] /= ph;
            break;
        }
    return o;
}

enum Kind { EMPTY, ZERO_H, ONE_H, TWO_H };

struct Pending {
    M2 m = ident();
    Kind kind = EMPTY;
    int x = 0;
    double theta = 0.0;
};

Pending make_zeroh(int x, double theta)
{
    theta = norm_angle(theta);
    Pending p;
    if (x == 0 && std::abs(norm_angle(theta)) <= kAtol) return p;
    p.m = x ? mul(pauli_x(), phase_m(theta)) : phase_m(theta);
    p.kind = ZERO_H;
    p.x = x;
    p.theta = theta;
    return p;
}

Pending classify(const M2 &m)
{
    Pending p;
    if (equiv_up_to_phase(m, ident())) return p;
    const M2 n = drop_phase(m);
    if (std::abs(n.a[1]) <= kAtol && std::abs(n.a[2]) <= kAtol)
        return make_zeroh(0, norm_angle(std::arg(n.a[3]) - std::arg(n.a[0])));
    if (std::abs(n.a[0]) <= kAtol && std::abs(n.a[3]) <= kAtol) {
        const cd base = m.a[2];
        if (std::abs(base) > kAtol) {
            const cd ph = base / std::abs(base);
            return make_zeroh(1, norm_angle(std::arg(m.a[1] / ph) - std::arg(m.a[2] / ph)));
        }
    }
    const double r2 = 1.0 / std::sqrt(2.0);
    bool halves = true;
    for (int k = 0; k < 4; k++) halves = halves && std::abs(std::abs(n.a[k]) - r2) <= 1e-8 + kRtol * r2;
    if (halves && std::abs(n.a[0]) > kAtol) {
        const cd base = n.a[0];
        const double near_t = norm_angle(std::arg(n.a[2]) - std::arg(base));
        const double far_t = norm_angle(std::arg(n.a[1]) - std::arg(base));
        const cd expect11 = -std::polar(1.0, near_t + far_t) * base;
        if (std::abs(n.a[3] - expect11) <= 1e-8) {
            p.m = mul(mul(phase_m(near_t), had()), phase_m(far_t));
            p.kind = ONE_H;
            return p;
        }
    }
    p.m = m;
    p.kind = TWO_H;
    return p;
}

bool exact_h(const Pending &p) { return p.kind == ONE_H && equiv_up_to_phase(p.m, had()); }

M2 gate_matrix(const zxh_gate &g)
{
    cd u[4];
    switch (g.type) {
    case ZXH_GATE_Z: return M2{{1.0, 0.0, 0.0, -1.0}};
    case ZXH_GATE_RZ: return M2{{std::polar(1.0, -0.5 * g.theta), 0.0, 0.0, std::polar(1.0, 0.5 * g.theta)}};
    case ZXH_GATE_P: return M2{{1.0, 0.0, 0.0, std::polar(1.0, g.theta)}};
    case ZXH_GATE_X: return pauli_x();
    case ZXH_GATE_H: return had();
    case ZXH_GATE_U3: zxh::u3_matrix(g.theta, g.lambda, g.phi, u); break;
    case ZXH_GATE_RX: zxh::u3_matrix(g.theta, kPi / 2.0, -kPi / 2.0, u); break;
    default: return ident();
    }
    return M2{{u[0], u[1], u[2], u[3]}};
}

bool single_qubit(uint32_t t)
{
    return t == ZXH_GATE_Z || t == ZXH_GATE_RZ || t == ZXH_GATE_P || t == ZXH_GATE_X || t == ZXH_GATE_H ||
           t == ZXH_GATE_U3 || t == ZXH_GATE_RX;
}

zxh_gate rec(uint32_t type, uint32_t cq, uint32_t q, double th = 0.0, double la = 0.0, double ph = 0.0)
{
    zxh_gate g;
    g.type = type;
    g.cq = cq;
    g.q = q;
    g.reserved = 0;
    g.theta = th;
    g.lambda = la;
    g.phi = ph;
    return g;
}

struct Scheduler {
    std::vector<Pending> pend;
    std::vector<zxh_gate> out;
    bool boundary = true;

    // U3(theta, phi, lambda) angles of m up to a global phase: theta from the
    // magnitudes, the phases from the entries that carry the weight
    void emit_u(uint32_t q, const M2 &m)
    {
        const double c = std::abs(m.a[0]), s = std::abs(m.a[2]);
        const double theta = 2.0 * std::atan2(s, c);
        const double a = std::arg(m.a[0]);
        const double phi = std::arg(m.a[2]) - a;
        const double lam = c >= s ? std::arg(m.a[3]) - a - phi : std::arg(-m.a[1]) - a;
        out.push_back(rec(ZXH_GATE_U3, 0, q, theta, norm_angle(lam), norm_angle(phi)));
    }

    void flush(uint32_t q)
    {
        Pending &p = pend[q];
        switch (p.kind) {
        case EMPTY: return;
        case ZERO_H:
            if (std::abs(norm_angle(p.theta)) > kAtol) out.push_back(rec(ZXH_GATE_RZ, 0, q, norm_angle(p.theta)));
            if (p.x) out.push_back(rec(ZXH_GATE_X, 0, q));
            break;
        case ONE_H:
            if (exact_h(p)) out.push_back(rec(ZXH_GATE_H, 0, q));
            else emit_u(q, p.m);
            break;
        case TWO_H: emit_u(q, p.m); break;
        }
        p = Pending();
    }

    void flush_all()
    {
        for (uint32_t q = 0; q < pend.size(); q++) flush(q);
    }

    void absorb(uint32_t q, const M2 &m)
    {
        pend[q] = classify(mul(m, pend[q].m));
        if (!boundary) flush(q);
    }

    void cx(uint32_t c, uint32_t t)
    {
        if (!boundary) {
            flush(c);
            flush(t);
            out.push_back(rec(ZXH_GATE_CX, c, t));
            return;
        }
        for (uint32_t q : {c, t})
            if (pend[q].kind != EMPTY && !exact_h(pend[q])) flush(q);
        if (exact_h(pend[c]) && exact_h(pend[t])) {
            out.push_back(rec(ZXH_GATE_CX, t, c));
            return;
        }
        flush(c);
        flush(t);
        out.push_back(rec(ZXH_GATE_CX, c, t));
    }
};

}  // namespace

extern "C" int zxh_optimize_gates(size_t n, int level, const zxh_gate *gates, size_t count, zxh_gate *out,
                                  size_t capacity, size_t *out_count)
{
    using zxh::api::fail;
    if (!out_count || (count && !gates)) return fail(nullptr, ZXH_ERR_ARG, "null argument");
    if (n < 1 || n > 63) return fail(nullptr, ZXH_ERR_LIMIT, "n must be in 1..63");
    Scheduler s;
    s.pend.assign(n, Pending());
    s.boundary = level > 0;
    for (size_t i = 0; i < count; i++) {
        const zxh_gate &g = gates[i];
        const bool two = g.type == ZXH_GATE_CRZ || g.type == ZXH_GATE_CP || g.type == ZXH_GATE_CX;
        if (g.type != ZXH_GATE_BARRIER && g.q >= n) return fail(nullptr, ZXH_ERR_ARG, "gate target qubit out of range");
        if (two && (g.cq >= n || g.cq == g.q))
            return fail(nullptr, ZXH_ERR_ARG, "gate control qubit out of range or equal to the target");
        if (g.type == ZXH_GATE_BARRIER) {
            s.flush_all();
            s.out.push_back(rec(ZXH_GATE_BARRIER, 0, 0));
        } else if (single_qubit(g.type)) {
            s.absorb(g.q, gate_matrix(g));
        } else if (g.type == ZXH_GATE_CX) {
            s.cx(g.cq, g.q);
        } else if (g.type == ZXH_GATE_CP || g.type == ZXH_GATE_CRZ) {
            s.flush(g.cq);
            s.flush(g.q);
            s.out.push_back(g);
        } else {
            return fail(nullptr, ZXH_ERR_ARG, "unknown gate type " + std::to_string(g.type));
        }
    }
    s.flush_all();
    *out_count = s.out.size();
    if (!out) return ZXH_OK;  // size query
    if (s.out.size() > capacity) return fail(nullptr, ZXH_ERR_LIMIT, "output capacity below *out_count");
    for (size_t i = 0; i < s.out.size(); i++) out[i] = s.out[i];
    return ZXH_OK;
}
