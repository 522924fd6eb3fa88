// host.cpp -- host side of the B200-native ZXH path:
//   * AffineMap: the GF(2) address map with cached solutions.
//   * walk():    the reference execute() schedule (src/zxh/src/core/zxh.cpp:312-553)
//                turned into an operation list with real-address selectors.
//   * plan():    the operation list compiled into device passes (product init,
//                doubling, TMA-tiled passes with fused diagonal windows).
#include "host.h"

#include <algorithm>
#include <deque>
#include <cmath>
#include <map>
#include <memory>
#include <stdexcept>

namespace zxh {

// ---------------------------------------------------------------------------
// AffineMap

void AffineMap::reset(int n)
{
    n_ = n;
    m_ = 0;
    std::memset(rows_, 0, sizeof(rows_));
    b_ = 0;
    dirty_ = true;
}

void AffineMap::append_col(int q)
{
    rows_[q] |= 1ULL << m_;  // bitmat_t::append_col(e_q), bitmat.cpp:139-145
    m_++;
    dirty_ = true;
}

void AffineMap::row_xor(int dst, int src)
{
    rows_[dst] ^= rows_[src];  // bitmat_t::row_xor, bitmat.cpp:34-44
    dirty_ = true;
}

// One elimination of [A | I_n]: the reduced pivot row of column c carries, in its
// right half, which original rows sum to it. The solution of A x = e_q is then
// x_c = bit q of that combination, and e_q is in the span iff no zero row of the
// reduced left half has bit q set in its combination.
void AffineMap::refresh()
{
    uint64_t left[64], right[64];
    for (int i = 0; i < n_; i++) {
        left[i] = rows_[i];
        right[i] = 1ULL << i;
    }
    int pivot_of_col[64];
    int row = 0;
    for (int col = 0; col < m_; col++) {
        pivot_of_col[col] = -1;
        int piv = row;
        while (piv < n_ && !((left[piv] >> col) & 1)) piv++;
        if (piv >= n_) continue;
        std::swap(left[piv], left[row]);
        std::swap(right[piv], right[row]);
        for (int i = 0; i < n_; i++)
            if (i != row && ((left[i] >> col) & 1)) {
                left[i] ^= left[row];
                right[i] ^= right[row];
            }
        pivot_of_col[col] = row;
        row++;
    }
    uint64_t null_union = 0;
    for (int i = 0; i < n_; i++)
        if (left[i] == 0) null_union |= right[i];
    solvable_ = 0;
    for (int q = 0; q < n_; q++) {
        if ((null_union >> q) & 1) {
            sol_[q] = 0;
            continue;
        }
        uint64_t x = 0;
        for (int col = 0; col < m_; col++)
            if (pivot_of_col[col] >= 0 && ((right[pivot_of_col[col]] >> q) & 1)) x |= 1ULL << col;
        sol_[q] = x;
        solvable_ |= 1ULL << q;
    }
    dirty_ = false;
}

bool AffineMap::solve(int q, uint64_t &delta)
{
    if (dirty_) refresh();
    if (!((solvable_ >> q) & 1)) return false;
    delta = sol_[q];
    return true;
}

uint64_t AffineMap::virt(uint64_t real) const
{
    uint64_t v = 0;
    for (int q = 0; q < n_; q++)
        if (parity64(real & rows_[q]) ^ int((b_ >> q) & 1)) v |= 1ULL << q;
    return v;
}

// ---------------------------------------------------------------------------
// The execute() walk.

namespace {

constexpr double kPi = 3.14159265358979323846;
const double kU3BatchEps = double(1e-5f);  // zxh.cpp:29 (a float literal promoted to double)

cd phase(double a) { return std::exp(cd(0.0, a)); }

void build_u3(double th, double la, double ph, cd u[4])
{
    // build_u3_matrix, zxh.cpp:101-113
    const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
    const cd el = phase(la), ep = phase(ph), epl = phase(ph + la);
    u[0] = cd(c, 0.0);
    u[1] = -el * s;
    u[2] = ep * s;
    u[3] = epl * c;
}

struct Acc {
    bool active = false;
    cd u[4] = {cd(1, 0), cd(0, 0), cd(0, 0), cd(1, 0)};
};

bool close_val(cd a, cd b) { return std::abs(a - b) <= kU3BatchEps; }

bool is_identity(const Acc &a)
{
    return close_val(a.u[0], cd(1, 0)) && close_val(a.u[1], cd(0, 0)) && close_val(a.u[2], cd(0, 0)) &&
           close_val(a.u[3], cd(1, 0));
}

void acc_reset(Acc &a)
{
    a.active = false;
    a.u[0] = cd(1, 0);
    a.u[1] = cd(0, 0);
    a.u[2] = cd(0, 0);
    a.u[3] = cd(1, 0);
}

void left_mul(Acc &a, const cd n[4])
{
    // left_multiply_u3, zxh.cpp:144-156
    const cd o00 = a.u[0], o01 = a.u[1], o10 = a.u[2], o11 = a.u[3];
    a.u[0] = n[0] * o00 + n[1] * o10;
    a.u[1] = n[0] * o01 + n[1] * o11;
    a.u[2] = n[2] * o00 + n[3] * o10;
    a.u[3] = n[2] * o01 + n[3] * o11;
    a.active = !is_identity(a);
}

}  // namespace

void u3_matrix(double theta, double lambda, double phi, cd u[4]) { build_u3(theta, lambda, phi, u); }

int walk(const Gate *gates, size_t count, bool disable_x, int M, WalkState &ws, std::vector<Op> &ops, std::string &err)
{
    AffineMap &A = ws.map;
    const int N = A.n();
    std::vector<DiagTerm> window;
    Acc pend[64];
    int pend_count = 0;

    auto flush_window = [&]() {
        if (window.empty()) return;
        Op op;
        op.kind = Op::DIAG;
        op.m = ws.m;
        op.diag.swap(window);
        ops.push_back(std::move(op));
        window.clear();
    };

    auto flush_u3_batch = [&]() {
        if (pend_count == 0) return;
        Op op;
        op.kind = Op::U3BATCH;
        op.m = ws.m;
        for (int q = 0; q < N; q++) {
            if (!pend[q].active) continue;
            U3Op u;
            A.solve(q, u.delta);
            u.delta &= low_mask(ws.m);
            u.sel = A.selector(q);
            for (int k = 0; k < 4; k++) u.u[k] = pend[q].u[k];
            op.u3.push_back(u);
        }
        for (int q = 0; q < N; q++) acc_reset(pend[q]);
        pend_count = 0;
        if (!op.u3.empty()) ops.push_back(std::move(op));
    };

    // solve_expand (zxh.cpp:701-719): returns whether the state grew.
    auto solve_expand = [&](int q, uint64_t &delta) -> int {
        if (A.solve(q, delta)) return 0;
        if (ws.m + 1 > M) return -1;
        ws.m++;
        A.append_col(q);
        delta = 1ULL << (A.m() - 1);
        return 1;
    };

    // One pair op, after a possible expansion (apply_u3 / apply_x_explicit /
    // apply_cx_explicit, zxh.cpp:742-825).
    auto pair_op = [&](int q, const cd u[4], int ctrl_q) -> int {
        uint64_t d = 0;
        const int grew = solve_expand(q, d);
        if (grew < 0) return -1;
        U3Op op;
        op.delta = d & low_mask(ws.m);
        op.sel = A.selector(q);
        for (int k = 0; k < 4; k++) op.u[k] = u[k];
        if (ctrl_q >= 0) {
            op.has_ctrl = true;
            op.ctrl = A.selector(ctrl_q);
        }
        Op o;
        o.kind = grew ? Op::EXPAND : Op::U3BATCH;
        o.m = ws.m;
        o.u3.push_back(op);
        ops.push_back(std::move(o));
        return 0;
    };

    for (size_t gi = 0; gi < count;) {
        const Gate &g = gates[gi];
        if (g.type == G_H || g.type == G_U3) {
            flush_window();
            while (gi < count && (gates[gi].type == G_H || gates[gi].type == G_U3)) {
                const Gate &u = gates[gi];
                const bool isH = u.type == G_H;
                cd mat[4];
                build_u3(isH ? kPi / 2.0 : u.theta, isH ? kPi : u.lambda, isH ? 0.0 : u.phi, mat);
                uint64_t d;
                if (!A.solve(int(u.q), d)) {
                    flush_u3_batch();
                    if (pair_op(int(u.q), mat, -1) < 0) {
                        err = "gate needs a state larger than the size chosen at execute()";
                        return 5;
                    }
                    gi++;
                    continue;
                }
                Acc &a = pend[u.q];
                const bool was = a.active;
                if (!was) acc_reset(a), a.active = true;
                left_mul(a, mat);
                if (!was && a.active) pend_count++;
                else if (was && !a.active) pend_count--;
                gi++;
            }
            flush_u3_batch();
            continue;
        }
        switch (g.type) {
        case G_BARRIER:
            flush_window();
            break;
        case G_Z:
        case G_RZ: {
            const double th = g.type == G_Z ? kPi : g.theta;
            DiagTerm t;
            t.s0 = A.selector(int(g.q));
            t.theta = th;
            window.push_back(t);
            ws.gphase *= phase(-0.5 * th);  // zxh.cpp:477-493
            break;
        }
        case G_P: {
            DiagTerm t;
            t.s0 = A.selector(int(g.q));
            t.theta = g.theta;
            window.push_back(t);
            break;
        }
        case G_CP: {
            // All CP gates stay in the window: a CP whose selector straddles the
            // reference's 8-bit lane split is applied by the same pass (the
            // reference flushes and launches cp_kernel, zxh.cpp:526-541; the
            // product of diagonal factors is the same).
            DiagTerm t;
            t.s0 = A.selector(int(g.cq));
            t.s1 = A.selector(int(g.q));
            t.two = true;
            t.theta = g.theta;
            window.push_back(t);
            break;
        }
        case G_X:
            if (disable_x) {
                flush_window();
                const cd X[4] = {cd(0, 0), cd(1, 0), cd(1, 0), cd(0, 0)};
                if (pair_op(int(g.q), X, -1) < 0) {
                    err = "gate needs a state larger than the size chosen at execute()";
                    return 5;
                }
            } else {
                A.flip_b(int(g.q));
            }
            break;
        case G_CX:
            if (disable_x) {
                flush_window();
                const cd X[4] = {cd(0, 0), cd(1, 0), cd(1, 0), cd(0, 0)};
                if (pair_op(int(g.q), X, int(g.cq)) < 0) {
                    err = "gate needs a state larger than the size chosen at execute()";
                    return 5;
                }
            } else {
                A.row_xor(int(g.q), int(g.cq));
                A.b_xor(int(g.q), int(g.cq));
            }
            break;
        default:
            break;
        }
        gi++;
    }
    flush_window();
    return 0;
}

int calc_mem(const Gate *gates, size_t count, int n, bool disable_x)
{
    // zxh.cpp:648-681
    AffineMap A;
    A.reset(n);
    for (size_t i = 0; i < count; i++) {
        const Gate &g = gates[i];
        bool probe = false;
        if (g.type == G_X || g.type == G_CX) {
            if (!disable_x) {
                if (g.type == G_CX) A.row_xor(int(g.q), int(g.cq));
            } else {
                probe = true;
            }
        } else if (g.type == G_H || g.type == G_U3) {
            probe = true;
        }
        if (probe) {
            uint64_t d;
            if (!A.solve(int(g.q), d)) A.append_col(int(g.q));
        }
    }
    return A.m();
}

// ---------------------------------------------------------------------------
// Planner

namespace {

int64_t turns(double theta)
{
    // theta / (2 pi) as a 64-bit fixed-point fraction of a turn, wrapping mod 2^64.
    long double f = (long double)theta / (2.0L * 3.141592653589793238462643383279502884L);
    f -= floorl(f);
    long double s = f * 18446744073709551616.0L;  // 2^64
    if (s >= 18446744073709551616.0L) s -= 18446744073709551616.0L;
    return (int64_t)(uint64_t)s;
}

bool single_bit_or_zero(uint64_t a) { return (a & (a - 1)) == 0; }

int bit_index(uint64_t a) { return __builtin_ctzll(a); }

// Dense over the 64 address bits; an entry is live where its mask bit is set
// (so nothing is cleared up front). Visiting rows and columns in bit order gives
// the terms sorted by (i, j).
struct Poly {
    int64_t c0 = 0;
    int64_t lin[64];
    uint64_t lin_mask = 0;
    int64_t quad[64][64];  // [i][j], i < j
    uint64_t quad_mask[64];
    uint64_t quad_rows = 0;
    std::vector<DiagTerm> general;

    Poly() { std::memset(quad_mask, 0, sizeof(quad_mask)); }
    void add_lin(int i, int64_t c)
    {
        if (!((lin_mask >> i) & 1)) {
            lin[i] = 0;
            lin_mask |= 1ULL << i;
        }
        lin[i] += c;
    }
    void add_quad(int i, int j, int64_t c)
    {
        if (i == j) { add_lin(i, c); return; }
        if (i > j) std::swap(i, j);
        if (!((quad_mask[i] >> j) & 1)) {
            quad[i][j] = 0;
            quad_mask[i] |= 1ULL << j;
            quad_rows |= 1ULL << i;
        }
        quad[i][j] += c;
    }
};

// Expands a window into a polynomial over real address bits where every selector
// is a single bit (or constant), and keeps the rest as general terms.
void to_poly(const std::vector<DiagTerm> &terms, Poly &p)
{
    for (const DiagTerm &t : terms) {
        const bool simple = single_bit_or_zero(t.s0.alpha) && (!t.two || single_bit_or_zero(t.s1.alpha));
        if (!simple) {
            p.general.push_back(t);
            continue;
        }
        const int64_t th = turns(t.theta);
        // [S] = c + s*x_i with (c, s) = (beta, 1 - 2 beta); constant selector: s = 0.
        const int64_t c0 = t.s0.beta, s0 = t.s0.alpha ? (t.s0.beta ? -1 : 1) : 0;
        const int i0 = t.s0.alpha ? bit_index(t.s0.alpha) : -1;
        if (!t.two) {
            p.c0 += th * c0;
            if (s0) p.add_lin(i0, th * s0);
            continue;
        }
        const int64_t c1 = t.s1.beta, s1 = t.s1.alpha ? (t.s1.beta ? -1 : 1) : 0;
        const int i1 = t.s1.alpha ? bit_index(t.s1.alpha) : -1;
        p.c0 += th * c0 * c1;
        if (s1) p.add_lin(i1, th * c0 * s1);
        if (s0) p.add_lin(i0, th * c1 * s0);
        if (s0 && s1) p.add_quad(i0, i1, th * s0 * s1);
    }
}

template <typename T>
uint64_t put(std::vector<uint8_t> &blob, const T &v)
{
    uint64_t off = (blob.size() + 15) & ~uint64_t(15);
    blob.resize(off + sizeof(T));
    std::memcpy(blob.data() + off, &v, sizeof(T));
    return off;
}

template <typename T>
uint64_t put_vec(std::vector<uint8_t> &blob, const std::vector<T> &v)
{
    uint64_t off = (blob.size() + 15) & ~uint64_t(15);
    blob.resize(off + sizeof(T) * v.size() + 16);
    if (!v.empty()) std::memcpy(blob.data() + off, v.data(), sizeof(T) * v.size());
    return off;
}

uint64_t pext_pos(uint64_t x, const uint8_t *pos, int T)
{
    uint64_t r = 0;
    for (int k = 0; k < T; k++)
        if ((x >> pos[k]) & 1) r |= 1ULL << k;
    return r;
}

// Splits a 2x2 unitary into e^{i a} P(b) [[c, -s], [s, c]] P(d), P(t) = diag(1,
// e^{i t}): a = arg u00, b = arg u10 - a, and d from the larger of u11 (c >= s) and
// -u01, so every entry is reproduced from the phases of the entries that carry
// its weight (a tiny c or s makes the other phase ill-defined, not the product).
struct RealSplit {
    double c, s, a, b, d;
};

RealSplit real_split(const cd u[4])
{
    double c = std::abs(u[0]), s = std::abs(u[2]);
    const double r = std::hypot(c, s);
    c /= r;
    s /= r;
    RealSplit o;
    o.c = c;
    o.s = s;
    o.a = std::arg(u[0]);
    o.b = std::arg(u[2]) - o.a;
    o.d = c >= s ? std::arg(u[3]) - o.a - o.b : std::arg(-u[1]) - o.a;
    return o;
}

// Compiles one window for a tile geometry; returns its blob offset.
uint64_t compile_diag(std::vector<uint8_t> &blob, const std::vector<DiagTerm> &terms, const TileDev &g)
{
    const std::unique_ptr<Poly> pp(new Poly());
    to_poly(terms, *pp);
    const Poly &p = *pp;
    int coord_of_bit[64];
    for (int i = 0; i < 64; i++) coord_of_bit[i] = -1;
    for (uint32_t k = 0; k < g.T; k++) coord_of_bit[g.pos[k]] = int(k);

    DiagDev d;
    std::memset(&d, 0, sizeof(d));
    d.c0 = p.c0;
    std::vector<LinTerm> out_lin;
    std::vector<QuadTerm> out_quad, in_quad, cross;
    for (uint64_t lm = p.lin_mask; lm; lm &= lm - 1) {
        const int b = __builtin_ctzll(lm);
        const int64_t c = p.lin[b];
        if (c == 0) continue;
        const int k = coord_of_bit[b];
        if (k >= 0) d.lin_in[k] += c;
        else out_lin.push_back(LinTerm{uint32_t(b), 0, c});
    }
    for (uint64_t rows = p.quad_rows; rows; rows &= rows - 1) {
        const int i = __builtin_ctzll(rows);
        for (uint64_t cm = p.quad_mask[i]; cm; cm &= cm - 1) {
            const int j = __builtin_ctzll(cm);
            const int64_t c = p.quad[i][j];
            if (c == 0) continue;
            const int ki = coord_of_bit[i], kj = coord_of_bit[j];
            if (ki >= 0 && kj >= 0) in_quad.push_back(QuadTerm{uint32_t(std::min(ki, kj)), uint32_t(std::max(ki, kj)), c});
            else if (ki >= 0) cross.push_back(QuadTerm{uint32_t(ki), uint32_t(j), c});
            else if (kj >= 0) cross.push_back(QuadTerm{uint32_t(kj), uint32_t(i), c});
            else out_quad.push_back(QuadTerm{uint32_t(i), uint32_t(j), c});
        }
    }
    std::vector<GenTerm> gen;
    for (const DiagTerm &t : p.general) {
        GenTerm gt;
        gt.a1_t = pext_pos(t.s0.alpha, g.pos, int(g.T));
        gt.a1_out = t.s0.alpha & ~g.tile_mask;
        gt.b1 = uint32_t(t.s0.beta);
        if (t.two) {
            gt.a2_t = pext_pos(t.s1.alpha, g.pos, int(g.T));
            gt.a2_out = t.s1.alpha & ~g.tile_mask;
            gt.b2 = uint32_t(t.s1.beta);
        } else {
            gt.a2_t = 0;
            gt.a2_out = 0;
            gt.b2 = 1;  // constant-true second selector
        }
        gt.coef = turns(t.theta);
        gen.push_back(gt);
    }
    d.n_out_lin = uint32_t(out_lin.size());
    d.n_out_quad = uint32_t(out_quad.size());
    d.n_in_quad = uint32_t(in_quad.size());
    d.n_cross = uint32_t(cross.size());
    d.n_gen = uint32_t(gen.size());
    d.off_out_lin = put_vec(blob, out_lin);
    d.off_out_quad = put_vec(blob, out_quad);
    d.off_in_quad = put_vec(blob, in_quad);
    d.off_cross = put_vec(blob, cross);
    d.off_gen = put_vec(blob, gen);
    // cross terms grouped by tile coordinate for the lane-parallel per-tile sums
    std::stable_sort(cross.begin(), cross.end(), [](const QuadTerm &a, const QuadTerm &b) { return a.i < b.i; });
    std::vector<uint32_t> kidx(kMaxTileBits + 1, 0);
    for (const QuadTerm &t : cross) kidx[t.i + 1]++;
    for (int k = 0; k < kMaxTileBits; k++) kidx[k + 1] += kidx[k];
    d.off_cross = put_vec(blob, cross);
    d.off_kidx = put_vec(blob, kidx);
    return put(blob, d);
}

size_t count_general(const std::vector<DiagTerm> &w)
{
    size_t n = 0;
    for (const DiagTerm &t : w) n += !(single_bit_or_zero(t.s0.alpha) && (!t.two || single_bit_or_zero(t.s1.alpha)));
    return n;
}

// Compiles one window as a Walsh sum over tiles of 2^T amplitudes (walsh.cu): with
// [S] = (1 - (-1)^S) / 2 and q = theta / 4 in turns,
//   theta [S0]      = 2q - 2q s0 X(a0),
//   theta [S0] [S1] = q - q s0 X(a0) - q s1 X(a1) + q s0 s1 X(a0 ^ a1),
// s = (-1)^beta, X(a) = (-1)^parity(a & r); terms of equal mask merge and mask 0
// is the constant. All sums wrap modulo 2^64 turns, and 4q equals theta's turns to
// within rounding, so the phase of every amplitude is exact modulo a full turn.
uint64_t compile_walsh(std::vector<uint8_t> &blob, const std::vector<DiagTerm> &terms, int T)
{
    std::vector<std::pair<uint64_t, uint64_t>> acc;  // (mask, coefficient)
    acc.reserve(terms.size() * 4);
    uint64_t c0 = 0;
    auto add = [&](uint64_t mask, uint64_t v) {
        if (mask) acc.emplace_back(mask, v);
        else c0 += v;
    };
    for (const DiagTerm &t : terms) {
        const uint64_t q = uint64_t(turns(t.theta * 0.25));
        if (!t.two) {
            const uint64_t h = q << 1;
            add(0, h);
            add(t.s0.alpha, t.s0.beta ? h : uint64_t(0) - h);
            continue;
        }
        add(0, q);
        add(t.s0.alpha, t.s0.beta ? q : uint64_t(0) - q);
        add(t.s1.alpha, t.s1.beta ? q : uint64_t(0) - q);
        add(t.s0.alpha ^ t.s1.alpha, t.s0.beta == t.s1.beta ? q : uint64_t(0) - q);
    }
    std::sort(acc.begin(), acc.end(), [](const std::pair<uint64_t, uint64_t> &a, const std::pair<uint64_t, uint64_t> &b) {
        return a.first < b.first;
    });
    std::vector<WalshTermDev> out;
    for (size_t i = 0; i < acc.size();) {
        const uint64_t mask = acc[i].first;
        uint64_t w = 0;
        for (; i < acc.size() && acc[i].first == mask; i++) w += acc[i].second;
        if (w) out.push_back(WalshTermDev{(mask >> T) | ((mask & low_mask(T)) << kWalshGShift), int64_t(w)});
    }
    std::stable_sort(out.begin(), out.end(), [](const WalshTermDev &a, const WalshTermDev &b) {
        return (a.hi_g >> kWalshGShift) < (b.hi_g >> kWalshGShift);
    });
    WalshDev d;
    std::memset(&d, 0, sizeof(d));
    d.c0 = int64_t(c0);
    d.T = uint32_t(T);
    d.n_terms = uint32_t(out.size());
    d.off_terms = put_vec(blob, out);
    return put(blob, d);
}

U3Dev compile_u3(const U3Op &u, const TileDev &g)
{
    U3Dev d;
    std::memset(&d, 0, sizeof(d));
    d.delta_t = pext_pos(u.delta, g.pos, int(g.T));
    d.alpha_t = pext_pos(u.sel.alpha, g.pos, int(g.T));
    d.alpha_out = u.sel.alpha & ~g.tile_mask;
    d.beta = uint32_t(u.sel.beta);
    d.pivot = uint32_t(__builtin_ctzll(d.delta_t));
    if (u.has_ctrl) {
        d.has_ctrl = 1;
        d.ctrl_t = pext_pos(u.ctrl.alpha, g.pos, int(g.T));
        d.ctrl_out = u.ctrl.alpha & ~g.tile_mask;
        d.ctrl_beta = uint32_t(u.ctrl.beta);
    }
    for (int k = 0; k < 4; k++) {
        d.u[2 * k] = u.u[k].real();
        d.u[2 * k + 1] = u.u[k].imag();
    }
    return d;
}

TileDev make_geom(int m, int c, const std::vector<int> &dirs)
{
    TileDev g;
    std::memset(&g, 0, sizeof(g));
    g.m = uint32_t(m);
    g.c = uint32_t(c);
    g.h = uint32_t(dirs.size());
    g.T = g.c + g.h;
    uint64_t mask = low_mask(c);
    for (int k = 0; k < c; k++) g.pos[k] = uint8_t(k);
    for (size_t j = 0; j < dirs.size(); j++) {
        g.pos[c + j] = uint8_t(dirs[j]);
        mask |= 1ULL << dirs[j];
    }
    g.tile_mask = mask;
    g.free_mask = low_mask(m) & ~mask;
    g.ntiles = 1ULL << (m - int(g.T));
    return g;
}

}  // namespace

int64_t phase_turns(double theta) { return turns(theta); }

// ---------------------------------------------------------------------------
// General strided pass records (grow.cu)

bool GrowBuild::init(int eb, int mm, const std::vector<uint64_t> &rg)
{
    elem_bytes = eb;
    m = mm;
    regs = rg;
    gates.clear();
    sels.clear();
    terms[0].clear();
    terms[1].clear();
    std::memset(&dev, 0, sizeof(dev));
    const int F = grow_fixed_bits(eb);
    const int R = int(regs.size());
    if (R > 4 || m < F + R) return false;
    // reduced high parts with distinct leading bits: the items enumerate the
    // addresses with zeros at [0, F) and at those leading bits (coset representatives)
    std::vector<uint64_t> basis;  // sorted by leading bit, descending
    std::vector<int> piv;
    for (uint64_t d : regs) {
        uint64_t h = d >> F;
        for (uint64_t b : basis)
            if ((h >> (63 - __builtin_clzll(b))) & 1) h ^= b;
        if (!h) return false;  // dependent
        basis.push_back(h);
        std::sort(basis.begin(), basis.end(), [](uint64_t a, uint64_t b) { return a > b; });
        piv.push_back(63 - __builtin_clzll(h) + F);
    }
    std::sort(piv.begin(), piv.end());
    dev.m = uint32_t(m);
    dev.F = uint32_t(F);
    dev.R = uint32_t(R);
    for (int i = 0; i < R; i++) dev.piv[i] = uint8_t(piv[size_t(i)]);
    for (int k = 0; k < (1 << R); k++) {
        uint64_t D = 0;
        for (int i = 0; i < R; i++)
            if ((k >> i) & 1) D ^= regs[size_t(i)];
        dev.D[k] = D;
    }
    dev.nitems = 1ULL << (m - F - R);
    return true;
}

int GrowBuild::selector(const Sel &s)
{
    const uint64_t a = s.alpha & low_mask(m);
    for (size_t i = 0; i < sels.size(); i++)
        if (sels[i].alpha == a && sels[i].beta == uint32_t(s.beta)) return int(i);
    if (sels.size() >= size_t(kGrowMaxSel)) return -1;
    int kb = -1;
    for (size_t i = 0; i < regs.size(); i++)
        if (parity64(a & regs[i])) {
            if (kb >= 0) return -1;  // flips with two register coordinates
            kb = int(i);
        }
    GrowSelDev d;
    d.alpha = a;
    d.beta = uint32_t(s.beta);
    d.kbit = kb;
    sels.push_back(d);
    return int(sels.size()) - 1;
}

bool GrowBuild::all_real() const
{
    for (const GrowGateDev &g : gates)
        if (g.u[1] != 0.0 || g.u[3] != 0.0 || g.u[5] != 0.0 || g.u[7] != 0.0) return false;
    return true;
}

bool GrowBuild::add_gate(const U3Op &u, uint32_t gen, uint32_t slot, bool adjoint_matrix)
{
    if (gates.size() >= size_t(kGrowMaxGates) || u.has_ctrl || !u.delta) return false;
    const int F = int(dev.F);
    GrowGateDev g;
    std::memset(&g, 0, sizeof(g));
    const int sel = selector(u.sel);
    if (sel < 0) return false;
    int reg = -1;
    for (size_t i = 0; i < regs.size(); i++)
        if (regs[i] == u.delta) reg = int(i);
    if (reg >= 0) {
        if (sels[size_t(sel)].kbit != reg) return false;
        g.kind = 0;
        g.reg = uint32_t(reg);
    } else {
        if ((u.delta >> F) != 0 || sels[size_t(sel)].kbit != -1) return false;
        const int LV = elem_bytes == 8 ? 1 : 0;
        g.kind = 1;
        g.lane_x = uint32_t((u.delta >> LV) & 31);
        g.vec_x = LV ? uint32_t(u.delta & 1) : 0;
    }
    g.sel = uint32_t(sel);
    g.gen = gen;
    g.slot = slot;
    cd w[4] = {u.u[0], u.u[1], u.u[2], u.u[3]};
    if (adjoint_matrix) {  // U^dagger
        w[0] = std::conj(u.u[0]);
        w[1] = std::conj(u.u[2]);
        w[2] = std::conj(u.u[1]);
        w[3] = std::conj(u.u[3]);
    }
    for (int q = 0; q < 4; q++) {
        g.u[2 * q] = w[q].real();
        g.u[2 * q + 1] = w[q].imag();
    }
    gates.push_back(g);
    dev.ngates = uint32_t(gates.size());
    return true;
}

bool GrowBuild::add_window(int which, const std::vector<DiagTerm> &w, const std::vector<uint32_t> *gk,
                           const std::vector<uint32_t> *slot, bool inverse)
{
    const size_t mark = sels.size();
    std::vector<GrowTermDev> cls[3];
    for (size_t ti = 0; ti < w.size(); ti++) {
        const DiagTerm &t = w[ti];
        GrowTermDev d;
        std::memset(&d, 0, sizeof(d));
        const int s0 = selector(t.s0);
        const int s1 = t.two ? selector(t.s1) : 0xff;
        if (s0 < 0 || s1 < 0) {
            sels.resize(mark);
            return false;
        }
        d.s0 = uint8_t(s0);
        d.s1 = uint8_t(s1);
        d.coef = turns(inverse ? -t.theta : t.theta);
        if (gk) d.gk = uint8_t((*gk)[ti]);
        if (slot) d.slot = (*slot)[ti];
        const bool k0 = sels[size_t(s0)].kbit >= 0;
        const bool k1 = t.two && sels[size_t(s1)].kbit >= 0;
        if (t.two && s0 == s1) {  // S and S = S
            d.s1 = 0xff;
            cls[k0 ? 2 : 0].push_back(d);
        } else if (!t.two) {
            cls[k0 ? 2 : 0].push_back(d);
        } else {
            cls[(k0 || k1) ? 2 : 1].push_back(d);
        }
    }
    const size_t n = cls[0].size() + cls[1].size() + cls[2].size();
    if (n > size_t(kGrowMaxTerms)) {
        sels.resize(mark);
        return false;
    }
    terms[which].clear();
    for (int c = 0; c < 3; c++) terms[which].insert(terms[which].end(), cls[c].begin(), cls[c].end());
    dev.ncls[which][0] = uint32_t(cls[0].size());
    dev.ncls[which][1] = uint32_t(cls[0].size() + cls[1].size());
    dev.ncls[which][2] = uint32_t(n);
    return true;
}

// exp(2 pi i j / 1024), j = 0..1023, rounded from long double; computed once
const std::vector<double> &exp_table_f64()
{
    static const std::vector<double> tab = [] {
        const int nt = 1 << kExpTableBits;
        std::vector<double> t(2 * nt);
        for (int j = 0; j < nt; j++) {
            const long double a = 2.0L * 3.141592653589793238462643383279502884L * j / nt;
            t[2 * j] = double(cosl(a));
            t[2 * j + 1] = double(sinl(a));
        }
        return t;
    }();
    return tab;
}

const std::vector<float> &exp_table_f32()
{
    static const std::vector<float> tab(exp_table_f64().begin(), exp_table_f64().end());
    return tab;
}

void exp_table(int elem_bytes, std::vector<uint8_t> &bytes)
{
    // the table the planner's passes use
    const std::vector<double> &t = exp_table_f64();
    if (elem_bytes == 8) {
        std::vector<float> f(t.begin(), t.end());
        bytes.assign(reinterpret_cast<const uint8_t *>(f.data()), reinterpret_cast<const uint8_t *>(f.data() + f.size()));
    } else {
        bytes.assign(reinterpret_cast<const uint8_t *>(t.data()), reinterpret_cast<const uint8_t *>(t.data() + t.size()));
    }
}

void Plan::clear()
{
    blob.clear();
    passes.clear();
}

// Splits windows whose multi-bit-selector terms exceed what one diagonal step
// evaluates per amplitude; the pieces commute, so their order is free.
std::vector<Op> split_windows(const std::vector<Op> &ops, size_t max_general)
{
    std::vector<Op> out;
    out.reserve(ops.size());
    for (const Op &op : ops) {
        if (op.kind != Op::DIAG) {
            out.push_back(op);
            continue;
        }
        Op cur;
        cur.kind = Op::DIAG;
        cur.m = op.m;
        size_t ngen = 0;
        for (const DiagTerm &t : op.diag) {
            const bool simple = single_bit_or_zero(t.s0.alpha) && (!t.two || single_bit_or_zero(t.s1.alpha));
            if (!simple && ngen == max_general) {
                out.push_back(cur);
                cur.diag.clear();
                ngen = 0;
            }
            if (!simple) ngen++;
            cur.diag.push_back(t);
        }
        if (!cur.diag.empty()) out.push_back(cur);
    }
    return out;
}

int plan(const std::vector<Op> &ops_in, int elem_bytes, const PlanParams &pp, const WalkState &start, Plan &out,
         std::string &err, const std::vector<DiagTerm> *carry_in, std::vector<DiagTerm> *carry_out)
{
    out.clear();
    // windows with more than 32 general terms are split; otherwise the ops are used as given
    bool need_split = false;
    for (const Op &op : ops_in) {
        if (op.kind != Op::DIAG) continue;
        size_t ngen = 0;
        for (const DiagTerm &t : op.diag)
            ngen += !(single_bit_or_zero(t.s0.alpha) && (!t.two || single_bit_or_zero(t.s1.alpha)));
        need_split = need_split || ngen > 32;
    }
    // with the Walsh pass a window of any size stays whole: the passes that take at
    // most 32 general terms (tile prologues / epilogues) refuse bigger ones, which
    // then run standalone
    need_split = need_split && !pp.walsh;
    std::vector<Op> split_ops;
    if (need_split) split_ops = split_windows(ops_in, 32);
    const std::vector<Op> *opsp = need_split ? &split_ops : &ops_in;
    // A U3 batch that mixes gates whose pair delta is their own selector bit with
    // gates whose deltas span several bits (after CX transport) is split in two:
    // its gates act on distinct qubits and commute, so the single-bit ones run
    // first as span passes and the rest as general strided passes, instead of all
    // of them filling general strided passes.
    std::vector<Op> mixed_ops;
    if (pp.span && pp.real_split && !pp.grow_only && pp.span_mixed) {
        auto single = [](const U3Op &u) {
            return !u.has_ctrl && u.delta && !(u.delta & (u.delta - 1)) && u.sel.alpha == u.delta;
        };
        auto mixed = [&](const Op &op) {
            if (op.kind != Op::U3BATCH || op.m < span_tile_bits(elem_bytes)) return false;
            size_t nf = 0;
            for (const U3Op &u : op.u3) nf += single(u) ? 1 : 0;
            return nf >= 8 && nf < op.u3.size();
        };
        bool any = false;
        for (const Op &op : *opsp) any = any || mixed(op);
        if (any) {
            for (const Op &op : *opsp) {
                if (!mixed(op)) {
                    mixed_ops.push_back(op);
                    continue;
                }
                Op a = op, b = op;
                a.u3.clear();
                b.u3.clear();
                for (const U3Op &u : op.u3) (single(u) ? a : b).u3.push_back(u);
                mixed_ops.push_back(std::move(a));
                mixed_ops.push_back(std::move(b));
            }
            opsp = &mixed_ops;
        }
    }
    const std::vector<Op> &ops = *opsp;
    size_t i = 0;
    int m = start.m;

    // 1. Product-state prefix: expansions whose selector is constant on the old
    //    bits, starting from |0...0>, and diagonal windows made only of P phases on
    //    existing bits / constant selectors. The prefix is written in one pass.
    if (start.fresh && pp.grow_only) {
        Pass ps;
        ps.kind = Pass::INIT;
        ps.m = start.m;
        out.passes.push_back(ps);
    } else if (start.fresh) {
        ProductDev pd;
        std::memset(&pd, 0, sizeof(pd));
        cd a0(1.0, 0.0);
        cd v[64][2];
        int pm = start.init_bits;
        for (int b = 0; b < pm; b++) {
            v[b][0] = cd(1.0, 0.0);
            v[b][1] = cd(0.0, 0.0);
        }
        size_t j = 0;
        for (; j < ops.size(); j++) {
            const Op &op = ops[j];
            if (op.kind == Op::EXPAND) {
                const U3Op &u = op.u3[0];
                const uint64_t old_alpha = u.sel.alpha & low_mask(pm);
                const bool ctrl_const = !u.has_ctrl || (u.ctrl.alpha & low_mask(pm + 1)) == 0;
                if (old_alpha != 0 || !ctrl_const || op.m != pm + 1) break;
                if (u.has_ctrl && !u.ctrl.beta) {
                    // control constantly false: identity on old bits, new half zero
                    v[pm][0] = cd(1, 0);
                    v[pm][1] = cd(0, 0);
                } else if (u.sel.beta == 0) {
                    v[pm][0] = u.u[0];
                    v[pm][1] = u.u[2];
                } else {
                    v[pm][0] = u.u[3];
                    v[pm][1] = u.u[1];
                }
                pm++;
                continue;
            }
            if (op.kind == Op::DIAG) {
                bool ok = true;
                for (const DiagTerm &t : op.diag)
                    if (t.two && t.s0.alpha && t.s1.alpha) ok = false;
                    else if (!single_bit_or_zero(t.s0.alpha) || (t.two && !single_bit_or_zero(t.s1.alpha))) ok = false;
                if (!ok) break;
                // linear phases factor over bits
                for (const DiagTerm &t : op.diag) {
                    const Sel *var = nullptr;
                    bool cst = true;
                    if (t.s0.alpha) var = &t.s0;
                    else cst = cst && t.s0.beta;
                    if (t.two) {
                        if (t.s1.alpha) var = &t.s1;
                        else cst = cst && t.s1.beta;
                    }
                    if (!cst) continue;
                    const cd ph = std::exp(cd(0.0, t.theta));
                    if (!var) { a0 *= ph; continue; }
                    const int b = bit_index(var->alpha);
                    v[b][var->beta ? 0 : 1] *= ph;
                }
                continue;
            }
            break;
        }
        i = j;
        pd.m = uint32_t(pm);
        pd.c0 = uint32_t(std::min(pm, pp.product_table_bits));
        pd.c1 = uint32_t(std::min(pm - int(pd.c0), pp.product_table_bits));
        pd.c2 = uint32_t(pm - int(pd.c0) - int(pd.c1));
        if (pd.c2 > 16) {
            err = "product state larger than 2^(2*table bits + 16) amplitudes";
            return 5;
        }
        // three factor tables over consecutive bit ranges, computed in double
        std::vector<double> tab;
        auto add_table = [&](int lo, int bits, cd scale) {
            for (uint64_t y = 0; y < (1ULL << bits); y++) {
                cd acc = scale;
                for (int b = 0; b < bits; b++) acc *= ((y >> b) & 1) ? v[lo + b][1] : v[lo + b][0];
                tab.push_back(acc.real());
                tab.push_back(acc.imag());
            }
        };
        add_table(0, int(pd.c0), cd(1.0, 0.0));
        add_table(int(pd.c0), int(pd.c1), cd(1.0, 0.0));
        add_table(int(pd.c0 + pd.c1), int(pd.c2), a0);
        Pass ps;
        ps.kind = Pass::PRODUCT;
        ps.m = pm;
        ps.off = put(out.blob, pd);
        if (elem_bytes == 8) {
            std::vector<float> tf(tab.begin(), tab.end());
            ps.off2 = put_vec(out.blob, tf);
        } else {
            ps.off2 = put_vec(out.blob, tab);
        }
        out.passes.push_back(ps);
        m = pm;
    }

    const int tmax = elem_bytes == 8 ? pp.tile_bits_c64 : pp.tile_bits_c128;
    int last_tile_pass = -1;          // index of a tile pass that can take an epilogue
    const std::vector<DiagTerm> *held = nullptr;  // window waiting for the next tile pass
    std::deque<std::vector<DiagTerm>> owned;       // windows the planner builds (stable addresses)
    std::vector<DiagTerm> carry;                   // phases split off the last U3 batch, due after it
    if (carry_in) carry = *carry_in;               // (or left over by the previous plan)

    auto emit_tile = [&](int mm, int c, const std::vector<int> &dirs, const std::vector<const U3Op *> &u3s,
                         const std::vector<DiagTerm> *pro) {
        TileDev g = make_geom(mm, c, dirs);
        std::vector<StepDev> steps;
        if (pro) steps.push_back(StepDev{STEP_DIAG, 0, compile_diag(out.blob, *pro, g)});
        for (const U3Op *u : u3s) steps.push_back(StepDev{STEP_U3, 0, put(out.blob, compile_u3(*u, g))});
        Pass ps;
        ps.kind = Pass::TILE;
        ps.m = mm;
        ps.geom = g;
        ps.steps = steps;
        out.passes.push_back(ps);
        return int(out.passes.size()) - 1;
    };

    auto attach_epilogue = [&](int pidx, const std::vector<DiagTerm> &w) {
        Pass &ps = out.passes[pidx];
        ps.steps.push_back(StepDev{STEP_DIAG, 0, compile_diag(out.blob, w, ps.geom)});
    };

    uint64_t exp_off = 0;
    auto ensure_exp = [&]() {
        if (!exp_off) exp_off = elem_bytes == 8 ? put_vec(out.blob, exp_table_f32()) : put_vec(out.blob, exp_table_f64());
    };
    auto standalone_diag = [&](int mm, const std::vector<DiagTerm> &w) {
        ensure_exp();
        if (pp.grow_only && mm >= grow_fixed_bits(elem_bytes)) {  // a general strided pass with no gates
            Pass ps;
            ps.kind = Pass::GROW;
            ps.m = mm;
            if (ps.gb.init(elem_bytes, mm, std::vector<uint64_t>()) && ps.gb.add_window(0, w)) {
                ps.off2 = exp_off;
                out.passes.push_back(ps);
                return;
            }
        }
        const size_t ngen = count_general(w);
        if (pp.walsh && ngen >= size_t(pp.walsh_min_general) && mm >= walsh_tile_bits(elem_bytes)) {
            Pass ps;
            ps.kind = Pass::WALSH;
            ps.m = mm;
            ps.off = compile_walsh(out.blob, w, walsh_tile_bits(elem_bytes));
            ps.row_bits = int(reinterpret_cast<const WalshDev *>(out.blob.data() + ps.off)->n_terms);
            ps.off2 = exp_off;
            out.passes.push_back(ps);
            return;
        }
        const int rb = elem_bytes == 8 ? pp.diag_row_bits_c64 : pp.diag_row_bits_c128;
        const int T = std::min(mm, diag_tile_bits(elem_bytes, rb));
        TileDev g = make_geom(mm, T, std::vector<int>());
        // the diagonal pass evaluates at most 32 general terms per amplitude: a bigger
        // window (only below the Walsh pass's tile size) runs as several passes
        std::vector<Op> pieces;
        if (ngen > 32) {
            Op whole;
            whole.kind = Op::DIAG;
            whole.m = mm;
            whole.diag = w;
            pieces = split_windows(std::vector<Op>{whole}, 32);
        }
        const size_t npieces = pieces.empty() ? 1 : pieces.size();
        for (size_t k = 0; k < npieces; k++) {
            Pass ps;
            ps.kind = Pass::DIAG;
            ps.m = mm;
            ps.chunk_bits = pp.diag_chunk_bits;
            ps.row_bits = rb;
            ps.prefetch = elem_bytes == 8 ? pp.diag_prefetch_c64 : pp.diag_prefetch_c128;
            ps.geom = g;
            ps.off = compile_diag(out.blob, pieces.empty() ? w : pieces[k].diag, g);
            ps.off2 = exp_off;
            out.passes.push_back(ps);
        }
    };

    // Fuses a window into a fast pass as prologue (pre) or epilogue when it is
    // small enough for per-thread evaluation; returns false otherwise.
    auto fuse_fast = [&](Pass &ps, const std::vector<DiagTerm> &w, bool pre) -> bool {
        uint64_t &slot = ps.kind == Pass::ROW    ? (pre ? ps.row.off_pre : ps.row.off_post)
                         : ps.kind == Pass::SPAN ? (pre ? ps.span.off_pre : ps.span.off_post)
                                                 : (pre ? ps.fast.off_pre : ps.fast.off_post);
        if (slot) return false;
        const size_t mark = out.blob.size();
        const uint64_t off = compile_diag(out.blob, w, ps.geom);
        const DiagDev *d = reinterpret_cast<const DiagDev *>(out.blob.data() + off);
        if (d->n_gen != 0 || d->n_in_quad > uint32_t(pp.fast_fuse_quad)) {
            out.blob.resize(mark);
            return false;
        }
        ensure_exp();
        slot = off;
        ps.off2 = exp_off;
        return true;
    };

    // The carried phases as the last pass's epilogue, else on their own.
    auto flush_carry = [&]() {
        if (carry.empty()) return;
        const std::vector<DiagTerm> w = carry;
        carry.clear();
        if (last_tile_pass >= 0 &&
            (out.passes[last_tile_pass].kind == Pass::ROW || out.passes[last_tile_pass].kind == Pass::SPAN) &&
            out.passes[last_tile_pass].m == m && fuse_fast(out.passes[last_tile_pass], w, false)) {
            last_tile_pass = -1;
            return;
        }
        standalone_diag(m, w);
        last_tile_pass = -1;
    };

    const int tfast = fast_tile_bits(elem_bytes);
    const int rfast = fast_reg_bits(elem_bytes);
    const int clo_fast = std::max(elem_bytes == 8 ? 1 : 0,
                                  std::min(tfast - 1, elem_bytes == 8 ? pp.fast_contig_c64 : pp.fast_contig_c128));
    auto fast_ok = [&](const Op &op) {
        if (pp.grow_only || op.m < tfast) return false;
        for (const U3Op &u : op.u3)
            if (u.has_ctrl || !u.delta || (u.delta & (u.delta - 1)) || u.sel.alpha != u.delta) return false;
        return true;
    };

    // One fast pass over the gates (each with a single bit) in a tile made of
    // `c` contiguous bits plus `dirs`.
    auto emit_fast = [&](int mm, int c, std::vector<int> dirs, const std::vector<const U3Op *> &gs) {
        // pad the high directions so the tile has exactly tfast coordinates
        for (int b = c; int(dirs.size()) < tfast - c && b < mm; b++)
            if (std::find(dirs.begin(), dirs.end(), b) == dirs.end()) dirs.push_back(b);
        std::sort(dirs.begin(), dirs.end());
        Pass ps;
        ps.kind = Pass::FAST;
        ps.m = mm;
        ps.geom = make_geom(mm, c, dirs);
        std::memset(&ps.fast, 0, sizeof(ps.fast));
        int coord_of_bit[64];
        for (int b = 0; b < 64; b++) coord_of_bit[b] = -1;
        for (uint32_t k = 0; k < ps.geom.T; k++) coord_of_bit[ps.geom.pos[k]] = int(k);
        std::vector<int> regc;  // coordinates >= 5 carrying gates
        for (const U3Op *u : gs) {
            const int k = coord_of_bit[__builtin_ctzll(u->delta)];
            if (k >= 5) regc.push_back(k);
        }
        std::sort(regc.begin(), regc.end());
        const int nr = std::max<int>(1, (int(regc.size()) + rfast - 1) / rfast);
        ps.fast.R = uint32_t(rfast);
        ps.fast.nrounds = uint32_t(nr);
        for (int r = 0; r < nr; r++) {
            std::vector<int> rc(regc.begin() + std::min<size_t>(regc.size(), size_t(r) * rfast),
                                regc.begin() + std::min<size_t>(regc.size(), size_t(r + 1) * rfast));
            for (int k = 5; int(rc.size()) < rfast; k++)
                if (std::find(rc.begin(), rc.end(), k) == rc.end()) rc.push_back(k);
            std::vector<int> oc;
            for (int k = 5; k < tfast; k++)
                if (std::find(rc.begin(), rc.end(), k) == rc.end()) oc.push_back(k);
            for (int j = 0; j < rfast; j++) ps.fast.rounds[r].rc[j] = uint8_t(rc[j]);
            for (int j = 0; j < 3; j++) ps.fast.rounds[r].oc[j] = uint8_t(oc[j]);
        }
        for (const U3Op *u : gs) {
            FastGateDev fg;
            std::memset(&fg, 0, sizeof(fg));
            const int k = coord_of_bit[__builtin_ctzll(u->delta)];
            fg.coord = uint32_t(k);
            fg.round = 0;
            if (k >= 5) {
                const int idx = int(std::find(regc.begin(), regc.end(), k) - regc.begin());
                fg.round = uint32_t(idx / rfast);
            }
            fg.alpha_out = u->sel.alpha & ~ps.geom.tile_mask;
            fg.beta = uint32_t(u->sel.beta);
            for (int q = 0; q < 4; q++) {
                fg.u[2 * q] = u->u[q].real();
                fg.u[2 * q + 1] = u->u[q].imag();
            }
            ps.fgates.push_back(fg);
        }
        ps.fast.ngates = uint32_t(ps.fgates.size());
        out.passes.push_back(ps);
        return int(out.passes.size()) - 1;
    };

    const int fgrow = grow_fixed_bits(elem_bytes);
    const int rgrow = std::max(1, std::min(pp.grow_regs, grow_reg_bits(elem_bytes, false)));
    auto grow_ok = [&](const Op &op) {
        if (op.m < fgrow) return false;
        for (const U3Op &u : op.u3)
            if (u.has_ctrl || !u.delta) return false;
        return true;
    };
    // General strided passes for one batch: lane gates (delta inside the low
    // fgrow bits) ride in the first pass; the rest go in groups of up to rgrow
    // whose high parts are linearly independent.
    auto emit_grow = [&](const Op &op) -> bool {
        const int mm = op.m;
        std::vector<const U3Op *> lane, rest;
        for (const U3Op &u : op.u3) ((u.delta >> fgrow) == 0 ? lane : rest).push_back(&u);
        std::vector<std::vector<const U3Op *>> groups;
        std::vector<const U3Op *> remaining = rest;
        while (!remaining.empty()) {
            std::vector<const U3Op *> grp, defer;
            std::vector<uint64_t> basis;
            for (const U3Op *u : remaining) {
                if (int(grp.size()) == rgrow || mm < fgrow + int(grp.size()) + 1) {
                    defer.push_back(u);
                    continue;
                }
                uint64_t h = u->delta >> fgrow;
                for (uint64_t b : basis)
                    if ((h >> (63 - __builtin_clzll(b))) & 1) h ^= b;
                if (!h) {
                    defer.push_back(u);
                    continue;
                }
                basis.push_back(h);
                std::sort(basis.begin(), basis.end(), [](uint64_t a, uint64_t b) { return a > b; });
                grp.push_back(u);
            }
            if (grp.empty()) return false;
            groups.push_back(grp);
            remaining.swap(defer);
        }
        if (groups.empty()) groups.emplace_back();
        for (size_t gi = 0; gi < groups.size(); gi++) {
            std::vector<uint64_t> regs;
            for (const U3Op *u : groups[gi]) regs.push_back(u->delta);
            Pass ps;
            ps.kind = Pass::GROW;
            ps.m = mm;
            bool ok = ps.gb.init(elem_bytes, mm, regs);
            for (const U3Op *u : groups[gi]) ok = ok && ps.gb.add_gate(*u, 0, 0, false);
            if (gi == 0)
                for (const U3Op *u : lane) ok = ok && ps.gb.add_gate(*u, 0, 0, false);
            if (!ok) return false;
            out.passes.push_back(ps);
        }
        return true;
    };

    for (; i < ops.size(); i++) {
        const Op &op = ops[i];
        const std::vector<DiagTerm> *wd = op.kind == Op::DIAG ? &op.diag : nullptr;  // this op's window
        if (!carry.empty()) {
            if (op.kind == Op::DIAG) {  // diagonal windows commute: one window
                owned.push_back(carry);
                owned.back().insert(owned.back().end(), op.diag.begin(), op.diag.end());
                wd = &owned.back();
                carry.clear();
            } else if (op.kind == Op::U3BATCH && fast_ok(op) && !held && op.m == m) {
                owned.push_back(carry);  // the next batch's prologue
                held = &owned.back();
                carry.clear();
            } else if (op.kind == Op::U3BATCH && !held && last_tile_pass < 0) {
                // phases left over by the previous plan and no pass of this one yet to
                // take them as an epilogue: a window before the batch's first pass
                owned.push_back(carry);
                held = &owned.back();
                carry.clear();
            } else {
                flush_carry();
            }
        }
        if (op.kind == Op::U3BATCH && fast_ok(op)) {
            const int mm = op.m;
            // strided register passes: fixed gates (bits below frow: vector and lane
            // coordinates) plus up to rrow gates on register bits
            const int rwide = elem_bytes == 8 ? pp.row_wide_c64 : pp.row_wide_c128;
            const int frow = row_fixed_bits(elem_bytes, rwide), rrow = row_reg_bits(elem_bytes, rwide);
            const bool low_path = pp.low_pass && row_low_ok(elem_bytes, rwide) && mm >= frow + rrow;
            // real split: gate = e^{i a} P(b) rotation P(d); the P(d) of every gate
            // joins the prologue, P(b) and e^{i a} are carried to after the batch
            const bool split = low_path && pp.real_split;
            std::vector<U3Op> rot;
            std::vector<DiagTerm> pre_ph;
            if (split) {
                rot = op.u3;
                for (U3Op &u : rot) {
                    const RealSplit r = real_split(u.u);
                    u.u[0] = cd(r.c, 0.0);
                    u.u[1] = cd(-r.s, 0.0);
                    u.u[2] = cd(r.s, 0.0);
                    u.u[3] = cd(r.c, 0.0);
                    DiagTerm t;
                    t.s0 = u.sel;
                    t.theta = r.d;
                    pre_ph.push_back(t);
                    t.theta = r.b;
                    carry.push_back(t);
                    t.s0 = Sel{0, 1};  // constant selector: global phase
                    t.theta = r.a;
                    carry.push_back(t);
                }
                owned.push_back(held ? *held : std::vector<DiagTerm>());
                owned.back().insert(owned.back().end(), pre_ph.begin(), pre_ph.end());
                held = &owned.back();
            }
            std::vector<const U3Op *> gs;
            for (const U3Op &u : (split ? rot : op.u3)) gs.push_back(&u);
            std::sort(gs.begin(), gs.end(), [](const U3Op *a, const U3Op *b) { return a->delta < b->delta; });
            if (split && pp.span && mm >= span_tile_bits(elem_bytes)) {
                // span passes (span.cu): the gates on bits 0..T-1 in one low pass, the rest
                // in as few strided passes as take T - 3 each, spread evenly (fewer gates
                // per pass = longer contiguous runs, c = T - gates); the low pass runs
                // last, like the row passes' (the windows then land on the strided passes)
                const int T = span_tile_bits(elem_bytes);
                std::vector<const U3Op *> lowg, highg;
                for (const U3Op *u : gs) (__builtin_ctzll(u->delta) < T ? lowg : highg).push_back(u);
                const int first_pass = int(out.passes.size());
                auto emit_span = [&](const std::vector<const U3Op *> &grp, bool low) {
                    std::vector<int> dirs;
                    if (!low)
                        for (const U3Op *u : grp) dirs.push_back(__builtin_ctzll(u->delta));
                    const int c = low ? T : T - int(dirs.size());
                    Pass ps;
                    ps.kind = Pass::SPAN;
                    ps.m = mm;
                    ps.low = low ? 1 : 0;
                    ps.geom = make_geom(mm, c, dirs);
                    std::memset(&ps.span, 0, sizeof(ps.span));
                    ps.span.m = uint32_t(mm);
                    ps.span.c = uint32_t(c);
                    ps.span.low = low ? 1u : 0u;
                    for (int k2 = 0; k2 < T; k2++) {
                        ps.span.pos[k2] = ps.geom.pos[k2];
                        ps.span.rot[k2][0] = 0.0;
                        ps.span.rot[k2][1] = 0.0;
                    }
                    ps.span.tile_mask = ps.geom.tile_mask;
                    ps.span.ntiles = ps.geom.ntiles;
                    double scale = 1.0;
                    for (const U3Op *u : grp) {
                        const int b = __builtin_ctzll(u->delta);
                        const int coord = int(std::find(ps.geom.pos, ps.geom.pos + T, uint8_t(b)) - ps.geom.pos);
                        ps.span.gates |= 1u << coord;
                        // R = [[c, -s], [s, c]]; with beta = 1 the partner at bit value 0
                        // leads, which is R with s negated. One coefficient is factored out
                        // (the larger of |c|, |s|), the factors multiply into scale.
                        const double cc = u->u[0].real(), ss = u->sel.beta ? -u->u[2].real() : u->u[2].real();
                        if (std::fabs(cc) >= std::fabs(ss)) {
                            ps.span.rot[coord][0] = ss / cc;
                            ps.span.rot[coord][1] = 0.0;
                            scale *= cc;
                        } else {
                            ps.span.rot[coord][0] = cc / ss;
                            ps.span.rot[coord][1] = 1.0;
                            scale *= ss;
                        }
                    }
                    ps.span.scale = scale;
                    ps.prefetch = pp.span_land;
                    out.passes.push_back(ps);
                    last_tile_pass = int(out.passes.size()) - 1;
                };
                const int H = int(highg.size());
                const int per = T - std::max(3, std::min(8, pp.span_min_run));
                const int np = (H + per - 1) / per;
                std::vector<std::vector<const U3Op *>> groups(static_cast<size_t>(np));
                size_t kk = 0;
                for (int pi = 0; pi < np; pi++) {
                    // split 0: the larger groups on the lower bits; 2: on the higher bits
                    const int rank = pp.span_split == 2 ? np - 1 - pi : pi;
                    const size_t G = size_t(H / np + (rank < H % np ? 1 : 0));
                    if (pp.span_split == 1) {
                        for (int k2 = pi; k2 < H; k2 += np) groups[size_t(pi)].push_back(highg[size_t(k2)]);
                    } else {
                        groups[size_t(pi)].assign(highg.begin() + long(kk), highg.begin() + long(kk + G));
                    }
                    kk += G;
                }
                if (pp.span_order == 2) std::reverse(groups.begin(), groups.end());
                for (const auto &grp : groups) emit_span(grp, false);
                if (pp.span_order == 0) {
                    // the window before the batch rides on the first strided pass: the first
                    // one that runs two layouts, where there is one (a window on a
                    // three-layout pass cost more: 32 qubits complex64, 47.9 vs 51.5 ms per
                    // U3 + cz layer on B200)
                    for (int pi = first_pass; pi < first_pass + np; pi++)
                        if (span_layouts(elem_bytes, out.passes[size_t(pi)].span.gates, false, pp.span_land != 0) == 2) {
                            std::rotate(out.passes.begin() + first_pass, out.passes.begin() + pi,
                                        out.passes.begin() + pi + 1);
                            break;
                        }
                }
                if (!lowg.empty()) emit_span(lowg, true);
                if (held) {
                    if (!fuse_fast(out.passes[first_pass], *held, true)) {
                        // not fusable: run it on its own, before the batch
                        const std::vector<DiagTerm> w = *held;
                        std::vector<Pass> batch(out.passes.begin() + first_pass, out.passes.end());
                        out.passes.resize(first_pass);
                        standalone_diag(mm, w);
                        for (Pass &p2 : batch) out.passes.push_back(p2);
                        last_tile_pass = int(out.passes.size()) - 1;
                    }
                    held = nullptr;
                }
                m = mm;
                continue;
            }
            auto emit_row = [&](const std::vector<const U3Op *> &fixed, const std::vector<const U3Op *> &grp, int low) {
                std::vector<int> rb;
                for (const U3Op *u : grp) rb.push_back(__builtin_ctzll(u->delta));
                // pad with the lowest free bits so every thread keeps 2^R rows in flight
                for (int b = frow; int(rb.size()) < rrow && b < mm; b++)
                    if (std::find(rb.begin(), rb.end(), b) == rb.end()) rb.push_back(b);
                std::sort(rb.begin(), rb.end());
                Pass ps;
                ps.kind = Pass::ROW;
                ps.m = mm;
                ps.geom = make_geom(mm, frow, rb);
                std::memset(&ps.row, 0, sizeof(ps.row));
                ps.row.m = uint32_t(mm);
                ps.row.F = uint32_t(frow);
                ps.row.R = uint32_t(rb.size());
                ps.row.ngates = uint32_t(fixed.size() + grp.size());
                for (size_t r = 0; r < rb.size(); r++) ps.row.rb[r] = uint8_t(rb[r]);
                ps.row.tile_mask = ps.geom.tile_mask;
                ps.row.nitems = 1ULL << (mm - frow - int(rb.size()));
                ps.wide = rwide;
                ps.low = low;
                ps.real = split ? 1 : 0;
                auto add = [&](const U3Op *u, int coord) {
                    FastGateDev fg;
                    std::memset(&fg, 0, sizeof(fg));
                    fg.coord = uint32_t(coord);
                    fg.alpha_out = u->sel.alpha & ~ps.geom.tile_mask;
                    fg.beta = uint32_t(u->sel.beta);
                    for (int q = 0; q < 4; q++) {
                        fg.u[2 * q] = u->u[q].real();
                        fg.u[2 * q + 1] = u->u[q].imag();
                    }
                    ps.fgates.push_back(fg);
                };
                for (const U3Op *u : fixed) add(u, __builtin_ctzll(u->delta));
                for (const U3Op *u : grp)
                    add(u, frow + int(std::find(rb.begin(), rb.end(), __builtin_ctzll(u->delta)) - rb.begin()));
                if (split) {
                    // real passes take a dense table: one slot per coordinate (all of
                    // them in the low pass, the register ones otherwise), identity
                    // where the pass has no gate
                    const int c0 = low ? 0 : frow, ns = low ? frow + int(rb.size()) : int(rb.size());
                    std::vector<FastGateDev> dense(static_cast<size_t>(ns));
                    for (int k2 = 0; k2 < ns; k2++) {
                        std::memset(&dense[size_t(k2)], 0, sizeof(FastGateDev));
                        dense[size_t(k2)].coord = uint32_t(c0 + k2);
                        dense[size_t(k2)].u[0] = 1.0;
                        dense[size_t(k2)].u[6] = 1.0;
                    }
                    for (const FastGateDev &fg : ps.fgates) dense[size_t(int(fg.coord) - c0)] = fg;
                    ps.fgates = dense;
                    ps.row.ngates = uint32_t(ns);
                }
                out.passes.push_back(ps);
                last_tile_pass = int(out.passes.size()) - 1;
            };
            size_t k = 0;
            const int first_pass = int(out.passes.size());
            std::vector<const U3Op *> lows, lgrp;  // the low pass: gates on the fixed bits + low_regs more
            if (low_path) {
                const int nreg = std::min(rrow, elem_bytes == 8 ? pp.low_regs_c64 : pp.low_regs_c128);
                while (k < gs.size() && (gs[k]->delta >> frow) == 0) lows.push_back(gs[k++]);
                if (!lows.empty())
                    while (k < gs.size() && int(lgrp.size()) < nreg) lgrp.push_back(gs[k++]);
                // with split gates the low pass runs last (gates on different bits
                // commute): the phase windows then ride in the strided passes,
                // which have issue slots to spare, and the low pass has none
                if (!lows.empty() && !split) emit_row(lows, lgrp, 1);
            } else {
                const int G = std::max(pp.fast_gates, frow);
                std::vector<const U3Op *> first;
                while (k < gs.size() && int(first.size()) < G && (gs[k]->delta >> tfast) == 0) first.push_back(gs[k++]);
                if (!first.empty()) last_tile_pass = emit_fast(mm, tfast, std::vector<int>(), first);
            }
            // the rest: strided register passes over the high bits
            while (k < gs.size()) {
                std::vector<const U3Op *> grp;
                while (k < gs.size() && int(grp.size()) < rrow) grp.push_back(gs[k++]);
                emit_row(std::vector<const U3Op *>(), grp, 0);
            }
            if (!lows.empty() && split) emit_row(lows, lgrp, 1);
            if (held) {
                if (!fuse_fast(out.passes[first_pass], *held, true)) {
                    // not fusable: run it on its own, before the batch
                    const std::vector<DiagTerm> w = *held;
                    Pass keep_last;
                    std::vector<Pass> batch(out.passes.begin() + first_pass, out.passes.end());
                    out.passes.resize(first_pass);
                    standalone_diag(mm, w);
                    for (Pass &p : batch) out.passes.push_back(p);
                    last_tile_pass = int(out.passes.size()) - 1;
                }
                held = nullptr;
            }
            m = mm;
            continue;
        }
        if (op.kind == Op::DIAG) {
            if (held) standalone_diag(m, *held), held = nullptr;
            // a window after a low pass waits for the next batch's first pass if there is one
            const bool next_u3 = i + 1 < ops.size() && ops[i + 1].kind == Op::U3BATCH && ops[i + 1].m == op.m;
            const bool spare_low = last_tile_pass >= 0 && out.passes[last_tile_pass].low && next_u3;
            if (!spare_low && last_tile_pass >= 0 &&
                (out.passes[last_tile_pass].kind == Pass::FAST || out.passes[last_tile_pass].kind == Pass::ROW ||
                 out.passes[last_tile_pass].kind == Pass::SPAN) &&
                out.passes[last_tile_pass].m == op.m && fuse_fast(out.passes[last_tile_pass], *wd, false)) {
                last_tile_pass = -1;
            } else if (last_tile_pass >= 0 && out.passes[last_tile_pass].kind == Pass::GROW &&
                       out.passes[last_tile_pass].m == op.m && out.passes[last_tile_pass].gb.dev.ncls[1][2] == 0 &&
                       out.passes[last_tile_pass].gb.add_window(1, *wd)) {
                ensure_exp();
                out.passes[last_tile_pass].off2 = exp_off;
                last_tile_pass = -1;
            } else if (last_tile_pass >= 0 && out.passes[last_tile_pass].kind == Pass::TILE &&
                       out.passes[last_tile_pass].m == op.m &&
                       out.passes[last_tile_pass].steps.size() < size_t(pp.max_steps) && count_general(*wd) <= 32) {
                attach_epilogue(last_tile_pass, *wd);
                last_tile_pass = -1;  // keep one epilogue window per pass
            } else if (next_u3) {
                held = wd;
            } else {
                standalone_diag(op.m, *wd);
                last_tile_pass = -1;
            }
            continue;
        }
        if (op.kind == Op::EXPAND) {
            if (held) standalone_diag(m, *held), held = nullptr;
            const U3Op &u = op.u3[0];
            ExpandDev e;
            std::memset(&e, 0, sizeof(e));
            e.m_old = uint32_t(op.m - 1);
            e.alpha = u.sel.alpha & low_mask(op.m - 1);
            e.beta = uint32_t(u.sel.beta);
            e.has_ctrl = u.has_ctrl ? 1 : 0;
            e.ctrl_alpha = u.ctrl.alpha & low_mask(op.m - 1);
            e.ctrl_beta = uint32_t(u.ctrl.beta);
            for (int k = 0; k < 4; k++) {
                e.u[2 * k] = u.u[k].real();
                e.u[2 * k + 1] = u.u[k].imag();
            }
            Pass ps;
            ps.kind = Pass::EXPAND;
            ps.m = op.m;
            ps.off = put(out.blob, e);
            out.passes.push_back(ps);
            m = op.m;
            last_tile_pass = -1;
            continue;
        }
        // U3BATCH with multi-bit deltas: general strided passes (grow.cu)
        if ((pp.grow || pp.grow_only) && grow_ok(op)) {
            const int mm = op.m;
            const size_t first = out.passes.size();
            if (emit_grow(op)) {
                if (held) {
                    GrowBuild &gb = out.passes[first].gb;
                    if (gb.add_window(0, *held)) {
                        ensure_exp();
                        out.passes[first].off2 = exp_off;
                    } else {
                        std::vector<Pass> batch(out.passes.begin() + long(first), out.passes.end());
                        out.passes.resize(first);
                        standalone_diag(mm, *held);
                        for (Pass &p2 : batch) out.passes.push_back(p2);
                    }
                    held = nullptr;
                }
                last_tile_pass = int(out.passes.size()) - 1;
                m = mm;
                continue;
            }
            out.passes.resize(first);
        }
        // U3BATCH: group pair ops into tiles.
        const int mm = op.m;
        const int cfull = std::min(mm, tmax);
        std::vector<const U3Op *> low, high;
        for (const U3Op &u : op.u3) ((u.delta >> cfull) == 0 ? low : high).push_back(&u);
        std::vector<std::pair<std::vector<int>, std::vector<const U3Op *>>> groups;  // (dirs, ops) ; dirs empty = low
        for (size_t k = 0; k < low.size(); k += size_t(pp.max_gates)) {
            std::vector<const U3Op *> gvec(low.begin() + k, low.begin() + std::min(low.size(), k + size_t(pp.max_gates)));
            groups.push_back({std::vector<int>(), gvec});
        }
        const int clo = std::min(cfull, pp.contig_bits);
        const int maxdirs = tmax - clo;
        std::vector<int> dirs;
        std::vector<const U3Op *> cur;
        std::vector<const U3Op *> direct;  // ops too wide for any tile
        auto close_high = [&]() {
            if (cur.empty()) return;
            std::sort(dirs.begin(), dirs.end());
            groups.push_back({dirs, cur});
            dirs.clear();
            cur.clear();
        };
        for (const U3Op *u : high) {
            std::vector<int> need;
            for (int b = clo; b < mm; b++)
                if ((u->delta >> b) & 1) need.push_back(b);
            if (int(need.size()) > maxdirs) {
                direct.push_back(u);
                continue;
            }
            std::vector<int> uni = dirs;
            for (int b : need)
                if (std::find(uni.begin(), uni.end(), b) == uni.end()) uni.push_back(b);
            if (int(uni.size()) > maxdirs || int(cur.size()) >= pp.max_gates) {
                close_high();
                uni = need;
            }
            dirs = uni;
            cur.push_back(u);
        }
        close_high();
        if (!direct.empty()) {
            // pair ops of one batch commute, so the wide ones go first; a held
            // window must still precede them.
            if (held) standalone_diag(mm, *held), held = nullptr;
            for (const U3Op *u : direct) {
                PairDev pd;
                std::memset(&pd, 0, sizeof(pd));
                pd.m = uint32_t(mm);
                pd.pivot = uint32_t(63 - __builtin_clzll(u->delta));
                pd.delta = u->delta;
                pd.alpha = u->sel.alpha;
                pd.beta = uint32_t(u->sel.beta);
                pd.has_ctrl = u->has_ctrl ? 1 : 0;
                pd.ctrl_alpha = u->ctrl.alpha;
                pd.ctrl_beta = uint32_t(u->ctrl.beta);
                for (int k = 0; k < 4; k++) {
                    pd.u[2 * k] = u->u[k].real();
                    pd.u[2 * k + 1] = u->u[k].imag();
                }
                Pass ps;
                ps.kind = Pass::PAIR;
                ps.m = mm;
                ps.off = put(out.blob, pd);
                out.passes.push_back(ps);
            }
            last_tile_pass = -1;
        }
        if (held && count_general(*held) > 32) {  // more general terms than a tile step evaluates
            standalone_diag(mm, *held);
            held = nullptr;
        }
        for (size_t k = 0; k < groups.size(); k++) {
            const bool lowgrp = groups[k].first.empty();
            const int c = lowgrp ? cfull : clo;
            const std::vector<DiagTerm> *pro = (k == 0) ? held : nullptr;
            last_tile_pass = emit_tile(mm, c, groups[k].first, groups[k].second, pro);
        }
        held = nullptr;
        m = mm;
    }
    if (carry_out) {
        *carry_out = carry;
        carry.clear();
    }
    flush_carry();
    if (held) standalone_diag(m, *held);

    // finalize step arrays
    for (Pass &ps : out.passes) {
        if (ps.kind == Pass::GROW) {
            GrowBuild &gb = ps.gb;
            gb.dev.nsel = uint32_t(gb.sels.size());
            gb.dev.off_gates = put_vec(out.blob, gb.gates);
            gb.dev.off_sel = put_vec(out.blob, gb.sels);
            gb.dev.off_terms[0] = put_vec(out.blob, gb.terms[0]);
            gb.dev.off_terms[1] = put_vec(out.blob, gb.terms[1]);
            ps.off = put(out.blob, gb.dev);
            ps.prefetch = (pp.grow_staged & 2) ? 1 : 0;
            continue;
        }
        if (ps.kind == Pass::ROW) {
            ps.row.off_gates = put_vec(out.blob, ps.fgates);
            ps.off = put(out.blob, ps.row);
            continue;
        }
        if (ps.kind == Pass::SPAN) {
            ps.real = 0;  // the kernel form for its windows
            for (const uint64_t ow : {ps.span.off_pre, ps.span.off_post}) {
                if (!ow) continue;
                const DiagDev *d = reinterpret_cast<const DiagDev *>(out.blob.data() + ow);
                const bool lin = d->n_in_quad == 0 && d->n_cross == 0 && d->n_out_quad == 0 && d->n_gen == 0;
                ps.real = std::max(ps.real, lin ? 1 : 2);
            }
            ps.off = put(out.blob, ps.span);
            continue;
        }
        if (ps.kind == Pass::FAST) {
            ps.fast.g = ps.geom;
            ps.fast.off_gates = put_vec(out.blob, ps.fgates);
            ps.off = put(out.blob, ps.fast);
            continue;
        }
        if (ps.kind != Pass::TILE) continue;
        ps.geom.nsteps = uint32_t(ps.steps.size());
        ps.geom.off_steps = put_vec(out.blob, ps.steps);
        ps.off = put(out.blob, ps.geom);
    }
    return 0;
}

}  // namespace zxh
