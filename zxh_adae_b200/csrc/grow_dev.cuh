// grow_dev.cuh -- device side of the general strided pass: shared by its own
// kernel (grow.cu) and the persistent batch kernel (batch.cu).
#pragma once

#include "core.h"
#include "dev.cuh"

#include <cuda_runtime.h>

namespace zxh {
namespace gdev {


template <typename E>
struct GrowCfg;
template <>
struct GrowCfg<float2> {
    using VT = float4;
    static constexpr int V = 2;
};
template <>
struct GrowCfg<double2> {
    using VT = double2;
    static constexpr int V = 1;
};

constexpr int kGrowAdjGates = 8;  // gates of one adjoint pass (per-thread FP64 accumulators)

template <typename E>
__device__ __forceinline__ E shfl_xor_c(E v, int m);
template <>
__device__ __forceinline__ float2 shfl_xor_c(float2 v, int m)
{
    return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
template <>
__device__ __forceinline__ double2 shfl_xor_c(double2 v, int m)
{
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

template <typename E, typename RT>
__device__ __forceinline__ E mad2(const RT *m, E a, E b)  // m[0..3] = (x re, x im, y re, y im): x a + y b
{
    E o;
    o.x = m[0] * a.x - m[1] * a.y + m[2] * b.x - m[3] * b.y;
    o.y = m[0] * a.y + m[1] * a.x + m[2] * b.y + m[3] * b.x;
    return o;
}

// One row vector of the state at amplitude address a (zeros in the lane bits);
// complex64 vectors hold two amplitudes whose order follows bit 0 of a. Loads and
// stores go through L2 only (.cg): in the persistent batch kernel another SM may
// have written the previous pass of the same state.
template <typename E>
__device__ __forceinline__ typename GrowCfg<E>::VT grow_load(const E *s, uint64_t a, int lane)
{
    using VT = typename GrowCfg<E>::VT;
    if constexpr (GrowCfg<E>::V == 2) {
        VT t = __ldcg(reinterpret_cast<const VT *>(s) + ((a >> 1) ^ uint64_t(lane)));
        if (a & 1) t = make_float4(t.z, t.w, t.x, t.y);
        return t;
    } else {
        return __ldcg(reinterpret_cast<const VT *>(s) + (a ^ uint64_t(lane)));
    }
}

template <typename E>
__device__ __forceinline__ void grow_store(E *s, uint64_t a, int lane, typename GrowCfg<E>::VT t)
{
    using VT = typename GrowCfg<E>::VT;
    if constexpr (GrowCfg<E>::V == 2) {
        if (a & 1) t = make_float4(t.z, t.w, t.x, t.y);
        __stcg(reinterpret_cast<VT *>(s) + ((a >> 1) ^ uint64_t(lane)), t);
    } else {
        __stcg(reinterpret_cast<VT *>(s) + (a ^ uint64_t(lane)), t);
    }
}

// Register gate on coordinate RR: rows j (bit RR clear) and j | 2^RR. REAL: the
// matrix has no imaginary parts (RY and the like), half the multiply-adds.
template <int RR, int NR, int V, bool ADJ, bool REAL, typename VT, typename RT>
__device__ __forceinline__ void grow_reg_gate(VT (&x)[NR], VT (&y)[NR], const RT (&m)[V][8], uint32_t orient,
                                              uint32_t gen, double &acc)
{
    using E = decltype(vget(x[0], 0));
    RT part = 0;  // this item's share of the gradient, in the state's precision; added to acc in FP64
#pragma unroll
    for (int j = 0; j < NR; j++) {
        if ((j >> RR) & 1) continue;
        constexpr int B = 1 << RR;
#pragma unroll
        for (int v = 0; v < V; v++) {
            const E lo = vget(x[j], v), hi = vget(x[j | B], v);
            if constexpr (ADJ) {
                const E llo = vget(y[j], v), lhi = vget(y[j | B], v);
                if (gen == 1) {  // Im<l|Y|p> = Re(conj(l1) p0) - Re(conj(l0) p1), |0> member = lo unless flipped
                    const RT t = (lhi.x * lo.x + lhi.y * lo.y) - (llo.x * hi.x + llo.y * hi.y);
                    part += ((orient >> v) & 1) ? -t : t;
                } else if (gen == 2) {  // Im<l|X|p> = Im(conj(l0) p1 + conj(l1) p0)
                    part += (llo.x * hi.y - llo.y * hi.x) + (lhi.x * lo.y - lhi.y * lo.x);
                }
                if constexpr (REAL) {
                    vset(y[j], v, rmad2(m[v][0], llo, m[v][2], lhi));
                    vset(y[j | B], v, rmad2(m[v][4], llo, m[v][6], lhi));
                } else {
                    vset(y[j], v, mad2(&m[v][0], llo, lhi));
                    vset(y[j | B], v, mad2(&m[v][4], llo, lhi));
                }
            }
            if constexpr (REAL) {
                vset(x[j], v, rmad2(m[v][0], lo, m[v][2], hi));
                vset(x[j | B], v, rmad2(m[v][4], lo, m[v][6], hi));
            } else {
                vset(x[j], v, mad2(&m[v][0], lo, hi));
                vset(x[j | B], v, mad2(&m[v][4], lo, hi));
            }
        }
    }
    if constexpr (ADJ) acc += double(part);
}

template <int R, int NR, int V, bool ADJ, bool REAL, typename VT, typename RT>
__device__ __forceinline__ void grow_reg_dispatch(int rr, VT (&x)[NR], VT (&y)[NR], const RT (&m)[V][8],
                                                  uint32_t orient, uint32_t gen, double &acc)
{
    switch (rr) {
    case 0: if constexpr (R > 0) grow_reg_gate<0, NR, V, ADJ, REAL>(x, y, m, orient, gen, acc); break;
    case 1: if constexpr (R > 1) grow_reg_gate<(R > 1 ? 1 : 0), NR, V, ADJ, REAL>(x, y, m, orient, gen, acc); break;
    case 2: if constexpr (R > 2) grow_reg_gate<(R > 2 ? 2 : 0), NR, V, ADJ, REAL>(x, y, m, orient, gen, acc); break;
    case 3: if constexpr (R > 3) grow_reg_gate<(R > 3 ? 3 : 0), NR, V, ADJ, REAL>(x, y, m, orient, gen, acc); break;
    default: break;
    }
}

// Window polynomial over the register row bits for one vector slot: K + sum_i
// k_i w_i + sum_{i<j} k_i k_j q_ij. Term classes (sorted on the host): [0, n1)
// single selector without row dependence, [n1, n2) two selectors without row
// dependence, [n2, n) the rest.
// pair coefficients q_ij, i < j, stored row by row
template <int R>
struct WinPoly {
    static constexpr int NQ = R * (R - 1) / 2 > 0 ? R * (R - 1) / 2 : 1;
    int64_t K;
    int64_t w[R > 0 ? R : 1];
    int64_t q[NQ];
};

template <int R>
__host__ __device__ constexpr int qidx(int i, int j)  // i < j
{
    return i * (2 * R - i - 1) / 2 + (j - i - 1);
}

template <int R>
__device__ __forceinline__ void add_w(WinPoly<R> &P, int kb, int64_t val)
{
#pragma unroll
    for (int i = 0; i < R; i++)
        if (i == kb) P.w[i] += val;
}

template <int R>
__device__ __forceinline__ void add_q(WinPoly<R> &P, int a, int b, int64_t val)
{
    const int i = min(a, b), j = max(a, b);
#pragma unroll
    for (int ii = 0; ii < R; ii++)
#pragma unroll
        for (int jj = ii + 1; jj < R; jj++)
            if (ii == i && jj == j) P.q[qidx<R>(ii, jj)] += val;
}

template <int R>
__device__ __forceinline__ void window_poly(WinPoly<R> &P, const GrowTermDev *t, uint32_t n1, uint32_t n2, uint32_t n,
                                            const int8_t *kb, uint64_t c)
{
    P.K = 0;
#pragma unroll
    for (int i = 0; i < R; i++) P.w[i] = 0;
#pragma unroll
    for (int i = 0; i < WinPoly<R>::NQ; i++) P.q[i] = 0;
    for (uint32_t q = 0; q < n1; q++)
        if ((c >> t[q].s0) & 1) P.K += t[q].coef;
    for (uint32_t q = n1; q < n2; q++)
        if ((c >> t[q].s0) & (c >> t[q].s1) & 1) P.K += t[q].coef;
    for (uint32_t q = n2; q < n; q++) {
        const GrowTermDev tt = t[q];
        const int c0 = int((c >> tt.s0) & 1), k0 = kb[tt.s0];
        if (tt.s1 == 0xff) {  // (c0 ^ k) = c0 + k (1 - 2 c0)
            if (c0) P.K += tt.coef;
            add_w(P, k0, c0 ? -tt.coef : tt.coef);
            continue;
        }
        const int c1 = int((c >> tt.s1) & 1), k1 = kb[tt.s1];
        if (k0 >= 0 && k1 >= 0) {
            if (c0 & c1) P.K += tt.coef;
            add_w(P, k0, int64_t(1 - 2 * c0) * int64_t(c1) * tt.coef);
            add_w(P, k1, int64_t(c0) * int64_t(1 - 2 * c1) * tt.coef);
            const int64_t qv = int64_t((1 - 2 * c0) * (1 - 2 * c1)) * tt.coef;
            if (k0 == k1) add_w(P, k0, qv);  // k * k = k: both selectors flip with the same row bit
            else add_q(P, k0, k1, qv);
        } else {
            const int cf = k0 >= 0 ? c1 : c0, cv = k0 >= 0 ? c0 : c1, kk = k0 >= 0 ? k0 : k1;
            if (cf) {
                if (cv) P.K += tt.coef;
                add_w(P, kk, cv ? -tt.coef : tt.coef);
            }
        }
    }
}

template <int R>
struct WinPoly32 {
    uint32_t K;
    uint32_t w[R > 0 ? R : 1];
    uint32_t q[WinPoly<R>::NQ];
};

template <int R>
__device__ __forceinline__ WinPoly32<R> to32(const WinPoly<R> &P)
{
    WinPoly32<R> o;
    o.K = turns32(P.K);
#pragma unroll
    for (int i = 0; i < R; i++) o.w[i] = turns32(P.w[i]);
#pragma unroll
    for (int i = 0; i < WinPoly<R>::NQ; i++) o.q[i] = turns32(P.q[i]);
    return o;
}

// complex64: the window's phase in 32-bit turns per amplitude, summed per row from
// the row's bits (compile-time, so the polynomial stays in registers); applied to
// x and, when given, to y (adjoint passes: psi and lambda get the same phase)
template <int R, typename VT>
__device__ __forceinline__ void apply_poly32(VT (&x)[1 << R], const WinPoly32<R> (&P)[2], const float2 *s_exp,
                                             VT *y = nullptr)
{
    constexpr int NR = 1 << R;
#pragma unroll
    for (int g = 0; g < NR; g++) {
#pragma unroll
        for (int v = 0; v < 2; v++) {
            uint32_t a = P[v].K;
#pragma unroll
            for (int i = 0; i < R; i++) {
                if (!((g >> i) & 1)) continue;
                a += P[v].w[i];
#pragma unroll
                for (int j = i + 1; j < R; j++)
                    if ((g >> j) & 1) a += P[v].q[qidx<R>(i, j)];
            }
            const float2 ph = phase_factor32(s_exp, a);
            vset(x[g], v, cmul(vget(x[g], v), ph));
            if (y) vset(y[g], v, cmul(vget(y[g], v), ph));
        }
    }
}

template <typename E, int R, int V, typename VT>
__device__ __forceinline__ void apply_poly(VT (&x)[1 << R], const WinPoly<R> (&P)[V], const E *s_exp,
                                           VT *y = nullptr)
{
    constexpr int NR = 1 << R;
#pragma unroll
    for (int g = 0; g < NR; g++) {
#pragma unroll
        for (int v = 0; v < V; v++) {
            int64_t a = P[v].K;
#pragma unroll
            for (int i = 0; i < R; i++) {
                if (!((g >> i) & 1)) continue;
                a += P[v].w[i];
#pragma unroll
                for (int j = i + 1; j < R; j++)
                    if ((g >> j) & 1) a += P[v].q[qidx<R>(i, j)];
            }
            const E ph = phase_factor(s_exp, a);
            vset(x[g], v, cmul(vget(x[g], v), ph));
            if (y) vset(y[g], v, cmul(vget(y[g], v), ph));
        }
    }
}

template <typename E, int NT = kThreads>
struct GrowShared {
    using RT = typename ET<E>::R;
    E s_exp[1 << kExpTableBits];
    RT s_u[kGrowMaxGates][2][8];
    uint32_t s_g[kGrowMaxGates][4];  // kind | reg << 8, lane_x, vec_x, sel | gen << 8
    uint64_t s_D[16];
    uint64_t s_alpha[kGrowMaxSel];
    int8_t s_kb[kGrowMaxSel];
    GrowTermDev s_t[2][kGrowMaxTerms];
    double s_red[NT / 32];
    uint8_t s_mu[kGrowMaxSel];                     // selector bits inside the lane / vector bits
    uint64_t s_bmask;                              // selector betas
    double s_tacc[NT / 32][kGrowMaxTerms];         // adjoint windows: per-warp term gradients
    double s_gacc[NT / 32][kGrowAdjGates][32];     // adjoint gates: per-lane gradient sums (off the registers)
};

// Adjoint window gradients of one item, before the inverse phases are applied.
// Term q's gradient sum_a w_a (S_q(a) ? m1 : m0), w = Im(conj(lambda) psi), is
// split into terms whose selectors do not flip with the register rows (their
// sum over the warp comes from one Walsh-Hadamard transform of the per-lane row
// sums over the lane / vector bits: sum_x [P ^ mu.x] W(x) = (Wt +- What(mu)) / 2;
// lane q mod 32 owns term q) and the rest (per-thread sums over the rows, then a
// warp sum). Results are added to tacc[q] (one warp's row of the shared array).
template <int R, int V, typename VT>
__device__ __forceinline__ void adj_window_grad(const VT (&x)[1 << R], const VT (&y)[1 << R], const uint64_t (&c)[V],
                                                uint64_t pb, int lane, const GrowTermDev *t, const uint8_t *mu,
                                                const int8_t *kb, uint32_t n2, uint32_t n, double *tacc)
{
    constexpr int NR = 1 << R;
    constexpr int LV = (V == 2) ? 1 : 0;
    constexpr int RR = R > 0 ? R : 1;
    double W[V], Wi[RR][V], Wij[RR][RR][V];
#pragma unroll
    for (int v = 0; v < V; v++) {
        W[v] = 0.0;
#pragma unroll
        for (int i = 0; i < RR; i++) {
            Wi[i][v] = 0.0;
#pragma unroll
            for (int j = 0; j < RR; j++) Wij[i][j][v] = 0.0;
        }
    }
#pragma unroll
    for (int k = 0; k < NR; k++)
#pragma unroll
        for (int v = 0; v < V; v++) {
            const auto a = vget(x[k], v);
            const auto l = vget(y[k], v);
            const double w = double(l.x * a.y - l.y * a.x);  // Im(conj(lambda) psi), one conversion
            W[v] += w;
#pragma unroll
            for (int i = 0; i < R; i++) {
                if (!((k >> i) & 1)) continue;
                Wi[i][v] += w;
#pragma unroll
                for (int j = i + 1; j < R; j++)
                    if ((k >> j) & 1) Wij[i][j][v] += w;
            }
        }
    // row-independent terms: Walsh-Hadamard transform over the 2^F low positions
    double h[V];
#pragma unroll
    for (int v = 0; v < V; v++) h[v] = W[v];
    if constexpr (V == 2) {
        const double a = h[0], b = h[1];
        h[0] = a + b;
        h[1] = a - b;
    }
#pragma unroll
    for (int m = 1; m < 32; m <<= 1)
#pragma unroll
        for (int v = 0; v < V; v++) {
            const double o = __shfl_xor_sync(0xffffffffu, h[v], m);
            h[v] = (lane & m) ? (o - h[v]) : (h[v] + o);
        }
    const double Wt = __shfl_sync(0xffffffffu, h[0], 0);
    auto fetch = [&](uint32_t m) -> double {
        const int src = int(m >> LV) & 31;
        const double a = __shfl_sync(0xffffffffu, h[0], src);
        if constexpr (V == 2) {
            const double b = __shfl_sync(0xffffffffu, h[1], src);
            return (m & 1) ? b : a;
        }
        return a;
    };
    auto S = [&](int p, double wh) { return 0.5 * (Wt + (p ? wh : -wh)); };
    for (uint32_t r0 = 0; r0 < n2; r0 += 32) {
        const uint32_t q = r0 + uint32_t(lane);
        const bool live = q < n2;
        const GrowTermDev tt = t[live ? q : r0];
        const bool two = tt.s1 != 0xff;
        const uint32_t m0 = mu[tt.s0], m1 = two ? mu[tt.s1] : 0u;
        const int p0 = int((pb >> tt.s0) & 1), p1 = two ? int((pb >> tt.s1) & 1) : 0;
        const double f0 = fetch(m0), f1 = fetch(m1), f01 = fetch(m0 ^ m1);  // every lane shuffles
        const double sv = two ? 0.5 * (S(p0, f0) + S(p1, f1) - S(p0 ^ p1, f01)) : S(p0, f0);
        if (live && tt.gk) {
            const double g0 = tt.gk == 1 ? 1.0 : 0.0, g1 = tt.gk == 1 ? -1.0 : -2.0;
            tacc[q] += g0 * Wt + (g1 - g0) * sv;
        }
    }
    // row-dependent terms: per-thread sums over the rows, then a warp sum
    auto wsel = [&](int k, int v) {
        double r = 0.0;
#pragma unroll
        for (int i = 0; i < R; i++)
            if (i == k) r = Wi[i][v];
        return r;
    };
    auto wpair = [&](int a, int b, int v) {
        const int i = min(a, b), j = max(a, b);
        double r = 0.0;
#pragma unroll
        for (int ii = 0; ii < R; ii++)
#pragma unroll
            for (int jj = ii + 1; jj < R; jj++)
                if (ii == i && jj == j) r = Wij[ii][jj][v];
        return r;
    };
    for (uint32_t q = n2; q < n; q++) {
        const GrowTermDev tt = t[q];
        double g = 0.0;
        const double g0 = tt.gk == 1 ? 1.0 : 0.0, g1 = tt.gk == 1 ? -1.0 : -2.0;
#pragma unroll
        for (int v = 0; v < V; v++) {
            const int c0 = int((c[v] >> tt.s0) & 1), k0 = kb[tt.s0];
            double sv;
            if (tt.s1 == 0xff) {
                const double Wa = wsel(k0, v);
                sv = c0 ? W[v] - Wa : Wa;
            } else {
                const int c1 = int((c[v] >> tt.s1) & 1), k1 = kb[tt.s1];
                if (k0 >= 0 && k1 >= 0 && k0 != k1) {
                    const double Wa = wsel(k0, v), Wb = wsel(k1, v), Wab = wpair(k0, k1, v);
                    const double W11 = Wab, W10 = Wa - Wab, W01 = Wb - Wab, W00 = W[v] - Wa - Wb + Wab;
                    sv = ((c0 & c1) ? W00 : 0.0) + (((1 - c0) & c1) ? W10 : 0.0) + ((c0 & (1 - c1)) ? W01 : 0.0) +
                         (((1 - c0) & (1 - c1)) ? W11 : 0.0);
                } else if (k0 >= 0 && k1 >= 0) {  // both flip with the same row bit
                    const double Wa = wsel(k0, v);
                    sv = c0 == c1 ? (c0 ? W[v] - Wa : Wa) : 0.0;
                } else {
                    const int cd = k0 >= 0 ? c0 : c1, cf = k0 >= 0 ? c1 : c0, kd = k0 >= 0 ? k0 : k1;
                    const double Wa = wsel(kd, v);
                    sv = cf ? (cd ? W[v] - Wa : Wa) : 0.0;
                }
            }
            g += g0 * W[v] + (g1 - g0) * sv;
        }
        g = warp_sum_f64(g);
        if (lane == 0 && tt.gk) tacc[q] += g;
    }
}

// One general strided pass (or the part of it made of items first + warp,
// first + warp + step, ... below end) on the calling CTA. Every thread of the CTA
// calls it; it synchronises the CTA on entry and exit. REAL: every gate of the
// pass has a real matrix.
// Bytes of one row of a warp (32 lanes x 16-byte vectors), the unit of a staged copy.
constexpr uint32_t kGrowRowBytes = 512;

// Shared memory of the staged form: one mbarrier per warp (padded to 128 bytes),
// then per warp the rows of one item of each state.
template <int R, bool ADJ>
__host__ __device__ constexpr size_t grow_stage_bytes()
{
    return 128 + size_t(kThreads / 32) * (ADJ ? 2 : 1) * (size_t(1) << R) * kGrowRowBytes;
}

// PF (staged form): every warp keeps the rows of its next item on their way into
// shared memory (one TMA bulk copy per row, completing on the warp's mbarrier)
// while it works on the current one, so the loads of one item overlap the
// arithmetic and stores of the previous one without holding registers. stage is
// the dynamic shared memory laid out as grow_stage_bytes; a wait that gives up
// (after about a second) records kErrTimeout in status and ends the warp's loop.
// psi_src (optional): psi is read from there and written to psi (the adjoint
// sweep's first pass after a checkpoint reads the checkpoint instead of copying
// it back first); every amplitude is read before it is written, by its own warp.
// NT: threads of the CTA (a multiple of 32).
template <typename E, int R, bool ADJ, bool REAL = false, bool PF = false, int NT = kThreads>
__device__ __forceinline__ void grow_body(const uint8_t *__restrict__ blob, uint64_t poff, uint64_t toff,
                                          E *__restrict__ psi, E *__restrict__ lam, double *grads, uint64_t first,
                                          uint64_t step, uint64_t end, GrowShared<E, NT> &sm, uint8_t *stage = nullptr,
                                          DevStatus *status = nullptr, const E *psi_src = nullptr)
{
    const E *ps = psi_src ? psi_src : psi;
    using VT = typename GrowCfg<E>::VT;
    using RT = typename ET<E>::R;
    constexpr int V = GrowCfg<E>::V;
    constexpr int LV = (V == 2) ? 1 : 0;
    constexpr int F = 5 + LV;
    constexpr int NR = 1 << R;
    constexpr int WARPS = NT / 32;

    const GrowDev &p = *reinterpret_cast<const GrowDev *>(blob + poff);
    const GrowGateDev *gates = reinterpret_cast<const GrowGateDev *>(blob + p.off_gates);
    const GrowSelDev *sels = reinterpret_cast<const GrowSelDev *>(blob + p.off_sel);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t ngates = p.ngates, nsel = p.nsel;
    const bool win0 = p.ncls[0][2] != 0, win1 = p.ncls[1][2] != 0;

    auto &s_exp = sm.s_exp;
    auto &s_u = sm.s_u;
    auto &s_g = sm.s_g;
    auto &s_D = sm.s_D;
    auto &s_alpha = sm.s_alpha;
    auto &s_kb = sm.s_kb;
    auto &s_t = sm.s_t;
    auto &s_red = sm.s_red;
    __syncthreads();  // the shared tables may still be read by a previous call

    if (win0 || win1) {
        const E *tab = reinterpret_cast<const E *>(blob + toff);
        for (int i = tid; i < (1 << kExpTableBits); i += NT) s_exp[i] = tab[i];
    }
    for (int w = 0; w < 2; w++) {
        const GrowTermDev *tt = reinterpret_cast<const GrowTermDev *>(blob + p.off_terms[w]);
        for (uint32_t i = uint32_t(tid); i < p.ncls[w][2]; i += NT) s_t[w][i] = tt[i];
    }
    if (tid < int(ngates)) {
        const GrowGateDev &gg = gates[tid];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            s_u[tid][0][i] = RT(gg.u[i]);
            s_u[tid][1][i] = RT(gg.u[i ^ 6]);  // |1> member first: [[u11, u10], [u01, u00]]
        }
        s_g[tid][0] = gg.kind | (gg.reg << 8);
        s_g[tid][1] = gg.lane_x;
        s_g[tid][2] = gg.vec_x;
        s_g[tid][3] = gg.sel | (gg.gen << 8);
    }
    if (tid < NR) s_D[tid] = p.D[tid];
    if (tid < int(nsel)) {
        s_alpha[tid] = sels[tid].alpha;
        s_kb[tid] = int8_t(sels[tid].kbit);
        sm.s_mu[tid] = uint8_t(sels[tid].alpha & ((1u << F) - 1u));
    }
    if (tid == 0) {
        uint64_t bm = 0;
        for (uint32_t s = 0; s < nsel; s++) bm |= uint64_t(sels[s].beta & 1) << s;
        sm.s_bmask = bm;
    }
    if constexpr (ADJ) {
        for (uint32_t i = uint32_t(tid); i < uint32_t(WARPS) * kGrowMaxTerms; i += NT) (&sm.s_tacc[0][0])[i] = 0.0;
        for (uint32_t i = uint32_t(tid); i < uint32_t(WARPS) * kGrowAdjGates * 32; i += NT)
            (&sm.s_gacc[0][0][0])[i] = 0.0;
    }
    // lane part of every selector (with beta), per vector slot
    uint64_t lb[V];
#pragma unroll
    for (int v = 0; v < V; v++) {
        lb[v] = 0;
        const uint64_t e = (uint64_t(lane) << LV) | uint64_t(v);
        for (uint32_t s = 0; s < nsel; s++)
            lb[v] |= uint64_t(par64(sels[s].alpha & e) ^ int(sels[s].beta & 1)) << s;
    }
    // staged form: this warp's barrier and row buffers
    constexpr int NS = ADJ ? 2 : 1;
    [[maybe_unused]] uint64_t *wbar = nullptr;
    [[maybe_unused]] VT *wbuf = nullptr;
    if constexpr (PF) {
        wbar = reinterpret_cast<uint64_t *>(stage) + warp;
        wbuf = reinterpret_cast<VT *>(stage + 128) + size_t(warp) * NS * NR * 32;
        if (lane == 0) mbar_init(wbar, 1);
        fence_mbar_init();
    }
    __syncthreads();

    // first amplitude address of an item: the item's bits spread around the pivots
    auto item_base = [&](uint64_t item) {
        uint64_t r0 = item << F;
#pragma unroll
        for (int i = 0; i < R; i++) {
            const uint32_t b = p.piv[i];
            r0 = ((r0 >> b) << (b + 1)) | (r0 & ((1ULL << b) - 1ULL));
        }
        return r0;
    };
    // staged form: start the copies of an item's rows (lane j < NS * NR copies row
    // j % NR of state j / NR: the 512 contiguous bytes its lanes' vectors lie in)
    [[maybe_unused]] auto stage_item = [&](uint64_t item) {
        const uint64_t b0 = item_base(item);
        if (lane == 0) mbar_arrive_expect_tx(wbar, uint32_t(NS * NR) * kGrowRowBytes);
        __syncwarp();
        if (lane < NS * NR) {
            const int k = lane & (NR - 1);
            const E *src = (lane >= NR) ? lam : ps;
            const VT *row = reinterpret_cast<const VT *>(src) + (((b0 ^ s_D[k]) >> LV) & ~uint64_t(31));
            bulk_g2s(wbuf + size_t(lane) * 32, row, kGrowRowBytes, wbar);
        }
    };
    uint32_t taken = 0;  // items this warp has taken (the barrier's phase)
    if constexpr (PF) {
        if (first + uint64_t(warp) < end) stage_item(first + uint64_t(warp));
    }

    for (uint64_t item = first + uint64_t(warp); item < end; item += step, taken++) {
        const uint64_t r0 = item_base(item);
        VT x[NR], y[NR];
        if constexpr (PF) {
            if (!__all_sync(0xffffffffu, mbar_wait_bounded(wbar, taken & 1u))) {
                if (lane == 0) report(status, kErrTimeout, 9, item);
                (void)mbar_wait_bounded(wbar, taken & 1u);  // the copies may still be in flight
                break;
            }
#pragma unroll
            for (int k = 0; k < NR; k++) {
                const uint64_t a = r0 ^ s_D[k];
                const uint32_t slot = uint32_t((a >> LV) ^ uint64_t(lane)) & 31u;
                VT t = wbuf[k * 32 + slot];
                if constexpr (V == 2) {
                    if (a & 1) t = make_float4(t.z, t.w, t.x, t.y);
                }
                x[k] = t;
                if constexpr (ADJ) {
                    VT u = wbuf[(NR + k) * 32 + slot];
                    if constexpr (V == 2) {
                        if (a & 1) u = make_float4(u.z, u.w, u.x, u.y);
                    }
                    y[k] = u;
                }
            }
            __syncwarp();  // every lane has read the buffer before it is refilled
            if (item + step < end) stage_item(item + step);
        } else {
#pragma unroll
            for (int k = 0; k < NR; k++) {
                x[k] = grow_load(ps, r0 ^ s_D[k], lane);
                if constexpr (ADJ) y[k] = grow_load(lam, r0 ^ s_D[k], lane);
            }
        }
        // selector bits of this item: lane s takes selectors s and s + 32
        const bool p0 = lane < int(nsel) && par64(s_alpha[lane] & r0);
        const bool p1 = lane + 32 < int(nsel) && par64(s_alpha[lane + 32] & r0);
        const uint64_t P = uint64_t(__ballot_sync(0xffffffffu, p0)) | (uint64_t(__ballot_sync(0xffffffffu, p1)) << 32);
        uint64_t c[V];
#pragma unroll
        for (int v = 0; v < V; v++) c[v] = P ^ lb[v];

        if constexpr (!ADJ) {
            if (win0) {
                if constexpr (V == 2) {
                    WinPoly32<R> W[2];
#pragma unroll
                    for (int v = 0; v < 2; v++) {
                        WinPoly<R> t;
                        window_poly(t, s_t[0], p.ncls[0][0], p.ncls[0][1], p.ncls[0][2], s_kb, c[v]);
                        W[v] = to32(t);
                    }
                    apply_poly32<R>(x, W, reinterpret_cast<const float2 *>(s_exp));
                } else {
                    WinPoly<R> W[V];
#pragma unroll
                    for (int v = 0; v < V; v++)
                        window_poly(W[v], s_t[0], p.ncls[0][0], p.ncls[0][1], p.ncls[0][2], s_kb, c[v]);
                    apply_poly<E, R, V>(x, W, s_exp);
                }
            }
        }
        if constexpr (ADJ) {
            if (win1) {  // the window after the gates, undone first: gradients, then inverse phases
                adj_window_grad<R, V>(x, y, c, P ^ sm.s_bmask, lane, s_t[1], sm.s_mu, s_kb, p.ncls[1][1],
                                      p.ncls[1][2], sm.s_tacc[warp]);
                if constexpr (V == 2) {
                    WinPoly32<R> W[2];
#pragma unroll
                    for (int v = 0; v < 2; v++) {
                        WinPoly<R> t;
                        window_poly(t, s_t[1], p.ncls[1][0], p.ncls[1][1], p.ncls[1][2], s_kb, c[v]);
                        W[v] = to32(t);
                    }
                    apply_poly32<R>(x, W, reinterpret_cast<const float2 *>(s_exp), y);
                } else {
                    WinPoly<R> W[V];
#pragma unroll
                    for (int v = 0; v < V; v++)
                        window_poly(W[v], s_t[1], p.ncls[1][0], p.ncls[1][1], p.ncls[1][2], s_kb, c[v]);
                    apply_poly<E, R, V>(x, W, s_exp, y);
                }
            }
        }
        for (uint32_t g = 0; g < ngates; g++) {
            const uint32_t kr = s_g[g][0], sg = s_g[g][3];
            const uint32_t sel = sg & 0xff, gen = sg >> 8;
            uint32_t orient = 0;
#pragma unroll
            for (int v = 0; v < V; v++) orient |= uint32_t((c[v] >> sel) & 1) << v;
            RT m[V][8];
#pragma unroll
            for (int v = 0; v < V; v++)
#pragma unroll
                for (int i = 0; i < 8; i++) m[v][i] = s_u[g][(orient >> v) & 1][i];
            double ga = 0.0;
            if ((kr & 0xff) == 0) {
                grow_reg_dispatch<R, NR, V, ADJ, REAL>(int(kr >> 8), x, y, m, orient, gen, ga);
            } else {
                using EE = decltype(vget(x[0], 0));
                const int lx = int(s_g[g][1]), vx = int(s_g[g][2]);
                RT gpart = 0;
#pragma unroll
                for (int j = 0; j < NR; j++) {
                    EE nx[V], ny[V];
#pragma unroll
                    for (int v = 0; v < V; v++) {
                        const EE own = vget(x[j], v);
                        const EE src = vget(x[j], v ^ (V == 2 ? vx : 0));
                        const EE pt = lx ? shfl_xor_c(src, lx) : src;
                        if constexpr (REAL) nx[v] = rmad2(m[v][0], own, m[v][2], pt);
                        else nx[v] = mad2(&m[v][0], own, pt);
                        if constexpr (ADJ) {
                            const EE lown = vget(y[j], v);
                            const EE lsrc = vget(y[j], v ^ (V == 2 ? vx : 0));
                            const EE lpt = lx ? shfl_xor_c(lsrc, lx) : lsrc;
                            if (gen == 1) {  // own |0>: -Re(conj(l) p'), own |1>: +Re(conj(l) p')
                                const RT t = lown.x * pt.x + lown.y * pt.y;
                                gpart += ((orient >> v) & 1) ? t : -t;
                            } else if (gen == 2) {
                                gpart += lown.x * pt.y - lown.y * pt.x;
                            }
                            if constexpr (REAL) ny[v] = rmad2(m[v][0], lown, m[v][2], lpt);
                            else ny[v] = mad2(&m[v][0], lown, lpt);
                        }
                    }
#pragma unroll
                    for (int v = 0; v < V; v++) {
                        vset(x[j], v, nx[v]);
                        if constexpr (ADJ) vset(y[j], v, ny[v]);
                    }
                }
                if constexpr (ADJ) ga += double(gpart);
            }
            if constexpr (ADJ) {
                if (g < uint32_t(kGrowAdjGates)) sm.s_gacc[warp][g][lane] += ga;  // this lane's own slot
            }
        }
        if constexpr (!ADJ) {
            if (win1) {
                if constexpr (V == 2) {
                    WinPoly32<R> W[2];
#pragma unroll
                    for (int v = 0; v < 2; v++) {
                        WinPoly<R> t;
                        window_poly(t, s_t[1], p.ncls[1][0], p.ncls[1][1], p.ncls[1][2], s_kb, c[v]);
                        W[v] = to32(t);
                    }
                    apply_poly32<R>(x, W, reinterpret_cast<const float2 *>(s_exp));
                } else {
                    WinPoly<R> W[V];
#pragma unroll
                    for (int v = 0; v < V; v++)
                        window_poly(W[v], s_t[1], p.ncls[1][0], p.ncls[1][1], p.ncls[1][2], s_kb, c[v]);
                    apply_poly<E, R, V>(x, W, s_exp);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < NR; k++) {
            grow_store(psi, r0 ^ s_D[k], lane, x[k]);
            if constexpr (ADJ) grow_store(lam, r0 ^ s_D[k], lane, y[k]);
        }
    }
    if constexpr (ADJ) {
        if (win1) {
            __syncthreads();
            for (uint32_t q = uint32_t(tid); q < p.ncls[1][2]; q += NT) {
                if (!s_t[1][q].gk) continue;
                double t = 0.0;
                for (int w = 0; w < WARPS; w++) t += sm.s_tacc[w][q];
                atomicAdd(&grads[s_t[1][q].slot], t);
            }
        }
        // every gate's warp sums in one shared table, one barrier, one atomic per gate
        __syncthreads();  // s_tacc may still be read by the window reduction above
#pragma unroll
        for (int g = 0; g < kGrowAdjGates; g++) {
            if (uint32_t(g) >= ngates) break;
            const double v = warp_sum_f64(sm.s_gacc[warp][g][lane]);
            if (lane == 0) sm.s_tacc[warp][g] = v;
        }
        __syncthreads();
        if (tid < int(ngates) && tid < kGrowAdjGates && (s_g[tid][3] >> 8) != 0) {
            double t = 0.0;
            for (int w = 0; w < WARPS; w++) t += sm.s_tacc[w][tid];
            atomicAdd(&grads[gates[tid].slot], t);
        }
    }
}


}  // namespace gdev
}  // namespace zxh
