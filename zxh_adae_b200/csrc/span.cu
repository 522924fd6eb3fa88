// span.cu -- a U3 batch as span passes (sm_100a): up to 13 single-qubit gates per
// read-modify-write of the state, so a 30-qubit layer of U3 gates takes 3 passes
// (complex64 and complex128) instead of the reference's 30 sweeps
// (src/zxh/src/kernel/kernel_cuda.cu:390-423: one sweep per fused gate with a grid
// sync between) or the 5 (complex64) / 7 (complex128) register-row passes of
// u3pass.cu.
//
// A CTA (8 warps; two CTAs share an SM) owns a tile of 2^T amplitudes, 64 KiB: T =
// 13 for complex64 (32 amplitudes per thread in registers), T = 12 for complex128
// (16 per thread). The tile's coordinates k = 0..T-1 are the real bits pos[k]: bits
// 0..c-1 (runs of 2^c contiguous amplitudes) and then the gates' bits; the other
// real bits enumerate tiles. A thread's amplitudes differ in R coordinates (its
// register coordinates), its lane and warp fix the other 5 + 3. Layouts:
//   complex64  (R = 5)                              complex128 (R = 4)
//   A   regs 5..9,  lanes 0..4,  warps 10..12        regs 5..8,  lanes 0..4,  warps 9..11
//   A'  regs 0..4,  lanes 5..9,  warps 10..12        regs 0..3,  lanes 4..8,  warps 9..11
//   B   regs 3, 4, 10..12, lanes 0..2, 5, 6,         regs 4, 9..11, lanes 0..2, 5, 6,
//       warps 7..9                                   warps 3, 7, 8
// The tile is loaded in A (a warp reads 2^min(c,5) contiguous amplitudes per
// segment) and written from B (runs of 8), and the amplitudes move between layouts
// through one 64 KiB shared slab whose slots are XOR-swizzled so that every write
// and read of a layout change is conflict-free. In each layout the gates on its
// register coordinates are register updates. A pass runs A -> B when A and B hold
// all its gate coordinates (complex64 strided passes, complex128 ones with c >= 4),
// else A -> A' -> B (the low pass, complex128 strided passes with c = 3).
//
// Gates are the real rotations of the planner's real split (U = e^{ia} P(b) R P(d),
// host.cpp): complex64 takes one paired FP32 FMA per amplitude and gate, complex128
// two FP64 FMAs; their phases ride in the windows. A window before the gates
// (prologue) is applied in A, one after them (epilogue) in B: linear windows as one
// factor per thread times one per register pattern, others with in-tile quadratic
// terms by a Gray-code walk over the registers (32-bit turns for complex64, the
// full 64-bit turns for complex128).
#include "core.h"
#include "dev.cuh"
#include "host.h"
#include "sampler.h"

#include <algorithm>
#include <cuda_runtime.h>

namespace zxh {

namespace {

template <typename E>
struct SpanGeo;

// complex64: 8-byte slab slots; a bank pair is slot bits 0..3: bits 0, 1, 2, 3 XOR
// bits 6, 7, 8, 5. In each layout the lanes of a warp access (its register index
// fixed) differ in 5 coordinates whose images span bits 0..3, so each access is the
// minimum two wavefronts.
template <>
struct SpanGeo<float2> {
    static constexpr int T = 13, R = 5, W = 3;
    __host__ __device__ static constexpr int reg(int L, int r) { return L == 0 ? 5 + r : L == 1 ? r : (r < 2 ? 3 + r : T - 5 + r); }
    __host__ __device__ static constexpr int lane(int L, int b) { return L == 0 ? b : L == 1 ? 5 + b : (b < 3 ? b : 2 + b); }
    __host__ __device__ static constexpr int warp(int L, int w) { return L == 2 ? 7 + w : 10 + w; }
    __host__ __device__ static constexpr uint32_t slot(uint32_t t)
    {
        return t ^ ((t >> 6) & 1u) ^ (((t >> 7) & 1u) << 1) ^ (((t >> 8) & 1u) << 2) ^ (((t >> 5) & 1u) << 3);
    }
};

// complex128: 16-byte slots; a 16-byte access is served per 8 consecutive lanes,
// whose slots must differ in bits 0..2: bits 0, 1, 2 XOR bits 4, 5, 6. Lane bits
// 0..2 are coordinates 0..2 (A, B) or 4..6 (A'), and with the other coordinate of
// each pair fixed the map is one-to-one.
template <>
struct SpanGeo<double2> {
    static constexpr int T = 12, R = 4, W = 3;
    __host__ __device__ static constexpr int reg(int L, int r) { return L == 0 ? 5 + r : L == 1 ? r : (r == 0 ? 4 : 8 + r); }
    __host__ __device__ static constexpr int lane(int L, int b) { return L == 0 ? b : L == 1 ? 4 + b : (b < 3 ? b : 2 + b); }
    __host__ __device__ static constexpr int warp(int L, int w) { return L == 2 ? (w == 0 ? 3 : 6 + w) : 9 + w; }
    __host__ __device__ static constexpr uint32_t slot(uint32_t t) { return t ^ ((t >> 4) & 7u); }
};

constexpr int kSpanThreads = 256;  // 8 warps, two CTAs per SM (both geometries)

template <typename E>
__host__ __device__ constexpr int span_nr() { return 1 << SpanGeo<E>::R; }  // amplitudes per thread

template <typename E, int L>
__host__ __device__ constexpr uint32_t reg_index(int j)
{
    uint32_t t = 0;
    for (int r = 0; r < SpanGeo<E>::R; r++)
        if ((j >> r) & 1) t |= 1u << SpanGeo<E>::reg(L, r);
    return t;
}

template <typename E, int L>
__host__ __device__ constexpr uint32_t reg_mask() { return reg_index<E, L>(span_nr<E>() - 1); }

template <typename E, int L>
__device__ __forceinline__ uint32_t fixed_index(int lane, int warp)
{
    uint32_t t = 0;
#pragma unroll
    for (int b = 0; b < 5; b++) t |= uint32_t((lane >> b) & 1) << SpanGeo<E>::lane(L, b);
#pragma unroll
    for (int w = 0; w < SpanGeo<E>::W; w++) t |= uint32_t((warp >> w) & 1) << SpanGeo<E>::warp(L, w);
    return t;
}

// Real-address offset of tile index t.
template <typename E>
__device__ __forceinline__ uint64_t real_of(uint32_t t, const uint8_t *pos)
{
    uint64_t o = 0;
#pragma unroll
    for (int k = 0; k < SpanGeo<E>::T; k++)
        if ((t >> k) & 1) o |= 1ULL << pos[k];
    return o;
}

// The slot map is linear over GF(2): slot(a | b) = slot(a) ^ slot(b) for disjoint a, b.
template <typename E, int LA, int LB>
__device__ __forceinline__ void exchange(E (&x)[span_nr<E>()], E *slab, int lane, int warp)
{
    using G = SpanGeo<E>;
    const uint32_t sa = G::slot(fixed_index<E, LA>(lane, warp)), sb = G::slot(fixed_index<E, LB>(lane, warp));
    __syncthreads();  // the slab's previous reads are done
#pragma unroll
    for (int j = 0; j < span_nr<E>(); j++) slab[sa ^ G::slot(reg_index<E, LA>(j))] = x[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < span_nr<E>(); j++) x[j] = slab[sb ^ G::slot(reg_index<E, LB>(j))];
}

// The rotations of layout L's register coordinates that are in `mask`, each with
// one coefficient factored out (SpanDev): rot[k] = (tau, 0): x' = x - tau y,
// y' = y + tau x; (mu, 1): x' = mu x - y, y' = x + mu y.
template <int L>
__device__ __forceinline__ void rotate(float2 (&x)[32], const float2 *rot, uint32_t mask)
{
#pragma unroll
    for (int r = 0; r < SpanGeo<float2>::R; r++) {
        const int k = SpanGeo<float2>::reg(L, r);
        if (!((mask >> k) & 1)) continue;
        const float2 cm = rot[k];
        const float2 q = make_float2(cm.x, cm.x);
        if (cm.y == 0.0f) {
            const float2 nq = make_float2(-cm.x, -cm.x);
#pragma unroll
            for (int j = 0; j < 32; j++) {
                if ((j >> r) & 1) continue;
                const float2 lo = x[j], hi = x[j | (1 << r)];
                x[j] = __ffma2_rn(nq, hi, lo);
                x[j | (1 << r)] = __ffma2_rn(q, lo, hi);
            }
        } else {
#pragma unroll
            for (int j = 0; j < 32; j++) {
                if ((j >> r) & 1) continue;
                const float2 lo = x[j], hi = x[j | (1 << r)];
                x[j] = __ffma2_rn(q, lo, make_float2(-hi.x, -hi.y));
                x[j | (1 << r)] = __ffma2_rn(q, hi, lo);
            }
        }
    }
}

template <int L>
__device__ __forceinline__ void rotate(double2 (&x)[16], const double2 *rot, uint32_t mask)
{
#pragma unroll
    for (int r = 0; r < SpanGeo<double2>::R; r++) {
        const int k = SpanGeo<double2>::reg(L, r);
        if (!((mask >> k) & 1)) continue;
        const double2 cm = rot[k];
        const double q = cm.x;
        if (cm.y == 0.0) {
#pragma unroll
            for (int j = 0; j < 16; j++) {
                if ((j >> r) & 1) continue;
                const double2 lo = x[j], hi = x[j | (1 << r)];
                x[j] = make_double2(fma(-q, hi.x, lo.x), fma(-q, hi.y, lo.y));
                x[j | (1 << r)] = make_double2(fma(q, lo.x, hi.x), fma(q, lo.y, hi.y));
            }
        } else {
#pragma unroll
            for (int j = 0; j < 16; j++) {
                if ((j >> r) & 1) continue;
                const double2 lo = x[j], hi = x[j | (1 << r)];
                x[j] = make_double2(fma(q, lo.x, -hi.x), fma(q, lo.y, -hi.y));
                x[j | (1 << r)] = make_double2(fma(q, hi.x, lo.x), fma(q, hi.y, lo.y));
            }
        }
    }
}

// A window's phase at a thread's amplitudes in layout L for one tile, in a form
// that needs few registers while the amplitudes are live: linear windows give
// one factor per thread (times rowf[j] per register pattern); others give the
// thread's constant and its R register coefficients in turns (register x register
// terms come from qreg[j]): 32-bit turns for complex64, 64-bit for complex128.
template <typename E>
struct SpanWin;
template <>
struct SpanWin<float2> {
    float2 f;
    uint32_t a, w[5];
};
template <>
struct SpanWin<double2> {
    double2 f;
    int64_t a, w[4];
};

__device__ __forceinline__ uint32_t span_turns(int64_t th, const float2 *) { return turns32(th); }
__device__ __forceinline__ int64_t span_turns(int64_t th, const double2 *) { return th; }
__device__ __forceinline__ float2 span_phase(const float2 *tab, uint32_t th) { return phase_factor32(tab, th); }
__device__ __forceinline__ double2 span_phase(const double2 *tab, int64_t th) { return phase_factor(tab, th); }

template <typename E, int L, bool LINEAR>
__device__ __forceinline__ SpanWin<E> span_window_setup(const uint8_t *blob, const DiagDev &dd, const E *s_exp,
                                                        uint64_t base, int lane, int warp)
{
    using G = SpanGeo<E>;
    constexpr uint32_t RM = reg_mask<E, L>();
    const uint32_t fix = fixed_index<E, L>(lane, warp);
    const QuadTerm *cr = reinterpret_cast<const QuadTerm *>(blob + dd.off_cross);
    const LinTerm *ol = reinterpret_cast<const LinTerm *>(blob + dd.off_out_lin);
    const QuadTerm *oq = reinterpret_cast<const QuadTerm *>(blob + dd.off_out_quad);
    const uint32_t *kidx = reinterpret_cast<const uint32_t *>(blob + dd.off_kidx);
    // coefficient of each tile coordinate given the tile's out-of-tile bits (lane k)
    int64_t da = 0, K = 0;
    if (lane < G::T) {
        da = dd.lin_in[lane];
        for (uint32_t q = kidx[lane]; q < kidx[lane + 1]; q++) {
            const QuadTerm t = cr[q];
            if ((base >> t.j) & 1) da += t.coef;
        }
    }
    for (uint32_t q = uint32_t(lane); q < dd.n_out_lin; q += 32)
        if ((base >> ol[q].bit) & 1) K += ol[q].coef;
    for (uint32_t q = uint32_t(lane); q < dd.n_out_quad; q += 32) {
        const QuadTerm t = oq[q];
        if (((base >> t.i) & 1) && ((base >> t.j) & 1)) K += t.coef;
    }
    int64_t acc = warp_sum_i64(K) + dd.c0;
#pragma unroll
    for (int k = 0; k < G::T; k++) {
        const int64_t dk = __shfl_sync(0xffffffffu, da, k);
        if (!((RM >> k) & 1) && ((fix >> k) & 1)) acc += dk;
    }
    SpanWin<E> sw;
    if constexpr (LINEAR) {
        sw.f = phase_factor(s_exp, acc);
        return sw;
    }
    int64_t w[G::R];
#pragma unroll
    for (int r = 0; r < G::R; r++) w[r] = __shfl_sync(0xffffffffu, da, G::reg(L, r));
    // in-tile quadratic terms with a fixed coordinate set
    const QuadTerm *iq = reinterpret_cast<const QuadTerm *>(blob + dd.off_in_quad);
    for (uint32_t q = 0; q < dd.n_in_quad; q++) {
        const QuadTerm t = iq[q];
        const bool ri = (RM >> t.i) & 1, rj = (RM >> t.j) & 1;
        if (ri && rj) continue;  // register x register: in qreg
        if (!ri && !rj) {
            if (((fix >> t.i) & 1) && ((fix >> t.j) & 1)) acc += t.coef;
            continue;
        }
        const uint32_t other = ri ? t.j : t.i, reg = ri ? t.i : t.j;
        if (!((fix >> other) & 1)) continue;
#pragma unroll
        for (int r = 0; r < G::R; r++)
            if (uint32_t(G::reg(L, r)) == reg) w[r] += t.coef;
    }
    sw.a = span_turns(acc, s_exp);
#pragma unroll
    for (int r = 0; r < G::R; r++) sw.w[r] = span_turns(w[r], s_exp);
    return sw;
}

template <typename E, bool LINEAR>
__device__ __forceinline__ void span_window_apply(E (&x)[span_nr<E>()], const SpanWin<E> &sw, const E *rowf,
                                                  const int64_t *qreg, const E *s_exp)
{
    if constexpr (LINEAR) {
#pragma unroll
        for (int j = 0; j < span_nr<E>(); j++) x[j] = cmul(x[j], cmul(sw.f, rowf[j]));
    } else {
        auto a = sw.a;
#pragma unroll
        for (int jj = 0; jj < span_nr<E>(); jj++) {
            const int gj = jj ^ (jj >> 1);
            if (jj > 0) {
                const int fb = ctz_const(jj);
                if ((gj >> fb) & 1) a += sw.w[fb];
                else a -= sw.w[fb];
            }
            x[gj] = cmul(x[gj], span_phase(s_exp, a + span_turns(qreg[gj], s_exp)));
        }
    }
}

// Per-CTA tables of a span pass, filled once per launch by span_setup.
template <typename E, int WIN>
struct SpanShared {
    E exp[WIN ? (1 << kExpTableBits) : 1];  // WIN != 0
    E rot[kSpanBits];                       // (coefficient, form) per coordinate
    uint64_t roff[2][span_nr<E>()];         // real offsets of the register patterns: layout A (loads), B (stores)
    int64_t qreg[2][span_nr<E>()];          // window 0 in layout A, window 1 in layout B
    E rowf[2][span_nr<E>()];
    uint8_t pos[16];
};

template <typename E, int WIN>
__device__ __forceinline__ void span_setup(SpanShared<E, WIN> &sh, const SpanDev &p, const uint8_t *blob, uint64_t toff,
                                           int tid)
{
    constexpr int NR = span_nr<E>();
    if (tid < 16) sh.pos[tid] = p.pos[tid];
    if (tid < SpanGeo<E>::T) {
        sh.rot[tid].x = decltype(sh.rot[tid].x)(p.rot[tid][0]);
        sh.rot[tid].y = decltype(sh.rot[tid].y)(p.rot[tid][1]);
    }
    if constexpr (WIN != 0) {
        const E *tab = reinterpret_cast<const E *>(blob + toff);
        for (int i = tid; i < (1 << kExpTableBits); i += kSpanThreads) sh.exp[i] = tab[i];
    }
    __syncthreads();
    if (tid < 2 * NR) {
        const int L = tid / NR, j = tid % NR;
        sh.roff[L][j] = real_of<E>(L ? reg_index<E, 2>(j) : reg_index<E, 0>(j), sh.pos);
    }
    if (WIN && tid >= 2 * NR && tid < 4 * NR) {
        // tile-independent window parts: the register x register quadratic terms and,
        // for linear windows, the per-pattern factors
        const int d = (tid - 2 * NR) / NR, j = tid % NR;
        const uint64_t ow = d ? p.off_post : p.off_pre;
        int64_t qa = 0, lb = 0;
        if (ow) {
            const DiagDev &dd = *reinterpret_cast<const DiagDev *>(blob + ow);
            const uint32_t t = d ? reg_index<E, 2>(j) : reg_index<E, 0>(j);
            const QuadTerm *iq = reinterpret_cast<const QuadTerm *>(blob + dd.off_in_quad);
            for (uint32_t q = 0; q < dd.n_in_quad; q++)
                if (((t >> iq[q].i) & 1) && ((t >> iq[q].j) & 1)) qa += iq[q].coef;
            for (int k = 0; k < SpanGeo<E>::T; k++)
                if ((t >> k) & 1) lb += dd.lin_in[k];
        }
        sh.qreg[d][j] = qa;
        sh.rowf[d][j] = phase_factor(sh.exp, lb);
    }
    __syncthreads();
}

// First real address of a tile: the strided passes insert zeros at the tile's real
// bits (ascending); the low pass's tiles are contiguous.
template <typename E, bool LOW>
__device__ __forceinline__ uint64_t span_tile_base(uint64_t tile, const uint8_t *pos)
{
    if constexpr (LOW) return tile << SpanGeo<E>::T;
#pragma unroll
    for (int k = 0; k < SpanGeo<E>::T; k++) {
        const uint32_t b = pos[k];
        tile = ((tile >> b) << (b + 1)) | (tile & ((1ULL << b) - 1ULL));
    }
    return tile;
}

// The gates of each layout and where the rotations' common factor goes: into a
// linear window's per-thread factor where there is one, else one multiply before
// the store.
template <typename E>
struct SpanGates {
    uint32_t gA, gAp, gB;
    decltype(E{}.x) scale;
    bool scale_pre, scale_post, scale_end;
};

template <typename E, bool THREE, int WIN>
__device__ __forceinline__ SpanGates<E> span_gates(const SpanDev &p)
{
    SpanGates<E> g;
    const uint32_t gm = p.gates;
    g.gA = gm & reg_mask<E, 0>();
    g.gAp = THREE ? (gm & reg_mask<E, 1>() & ~g.gA) : 0u;
    g.gB = gm & reg_mask<E, 2>() & ~g.gA & ~g.gAp;
    g.scale = decltype(g.scale)(p.scale);
    g.scale_pre = WIN == 1 && p.off_pre != 0;
    g.scale_post = WIN == 1 && !g.scale_pre && p.off_post != 0;
    g.scale_end = !g.scale_pre && !g.scale_post;
    return g;
}

__device__ __forceinline__ void span_scale(float2 &x, float s) { x = __fmul2_rn(make_float2(s, s), x); }
__device__ __forceinline__ void span_scale(double2 &x, double s) { x = make_double2(x.x * s, x.y * s); }

// WIN: 0 no window, 1 windows with linear terms only, 2 any windows (quadratic
// terms; no multi-bit selectors). LOW: the tile is real bits 0..T-1. THREE: the
// layouts A, A', B (else A, B). Two CTAs share an SM; each works on one tile at a
// time: the windows' per-tile parts computed before the loads (few registers stay
// live across the tile), loads in layout A, exchanges through the slab, stores
// from layout B.
template <typename E, bool LOW, bool THREE, int WIN>
__global__ void __launch_bounds__(kSpanThreads, 2) span_kernel(const uint8_t *__restrict__ blob, uint64_t soff,
                                                              uint64_t toff, E *__restrict__ state)
{
    constexpr int NR = span_nr<E>();
    extern __shared__ __align__(16) unsigned char s_raw[];
    E *slab = reinterpret_cast<E *>(s_raw);  // 2^T slots
    __shared__ SpanShared<E, WIN> sh;

    const SpanDev &p = *reinterpret_cast<const SpanDev *>(blob + soff);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    span_setup(sh, p, blob, toff, tid);

    const uint64_t offA = real_of<E>(fixed_index<E, 0>(lane, warp), sh.pos);
    const uint64_t offB = real_of<E>(fixed_index<E, 2>(lane, warp), sh.pos);
    const SpanGates<E> g = span_gates<E, THREE, WIN>(p);
    const uint64_t ntiles = p.ntiles;

    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t base = span_tile_base<E, LOW>(tile, sh.pos);
        [[maybe_unused]] SpanWin<E> wpre, wpost;
        if constexpr (WIN != 0) {
            if (p.off_pre) {
                wpre = span_window_setup<E, 0, WIN == 1>(blob, *reinterpret_cast<const DiagDev *>(blob + p.off_pre),
                                                         sh.exp, base, lane, warp);
                if (g.scale_pre) span_scale(wpre.f, g.scale);
            }
            if (p.off_post) {
                wpost = span_window_setup<E, 2, WIN == 1>(blob, *reinterpret_cast<const DiagDev *>(blob + p.off_post),
                                                          sh.exp, base, lane, warp);
                if (g.scale_post) span_scale(wpost.f, g.scale);
            }
        }
        E x[NR];
        const E *src = state + base + offA;
#pragma unroll
        for (int j = 0; j < NR; j++) x[j] = __ldcs(src + sh.roff[0][j]);
        if constexpr (WIN != 0) {
            if (p.off_pre) span_window_apply<E, WIN == 1>(x, wpre, sh.rowf[0], sh.qreg[0], sh.exp);
        }
        rotate<0>(x, sh.rot, g.gA);
        if constexpr (THREE) {
            exchange<E, 0, 1>(x, slab, lane, warp);
            rotate<1>(x, sh.rot, g.gAp);
            exchange<E, 1, 2>(x, slab, lane, warp);
        } else {
            exchange<E, 0, 2>(x, slab, lane, warp);
        }
        rotate<2>(x, sh.rot, g.gB);
        if constexpr (WIN != 0) {
            if (p.off_post) span_window_apply<E, WIN == 1>(x, wpost, sh.rowf[1], sh.qreg[1], sh.exp);
        }
        if (g.scale_end) {
#pragma unroll
            for (int j = 0; j < NR; j++) span_scale(x[j], g.scale);
        }
        E *dst = state + base + offB;
#pragma unroll
        for (int j = 0; j < NR; j++) __stcs(dst + sh.roff[1][j], x[j]);
    }
}

template <typename E, bool LOW, bool THREE, int WIN>
cudaError_t launch_span(const uint8_t *dblob, uint64_t soff, uint64_t toff, uint64_t ntiles, E *state, int sms,
                        cudaStream_t st)
{
    auto kern = span_kernel<E, LOW, THREE, WIN>;
    const size_t smem = sizeof(E) << SpanGeo<E>::T;  // 64 KiB
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSpanThreads, smem);
    if (per_sm < 1) per_sm = 1;
    const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(sms) * uint64_t(per_sm))));
    kern<<<grid, kSpanThreads, smem, st>>>(dblob, soff, toff, state);
    return cudaGetLastError();
}

template <typename E, bool LOW, bool THREE>
cudaError_t launch_span_win(const uint8_t *dblob, uint64_t soff, uint64_t toff, uint64_t ntiles, int win, E *state,
                            int sms, cudaStream_t st)
{
    switch (win) {
    case 0: return launch_span<E, LOW, THREE, 0>(dblob, soff, toff, ntiles, state, sms, st);
    case 1: return launch_span<E, LOW, THREE, 1>(dblob, soff, toff, ntiles, state, sms, st);
    case 2: return launch_span<E, LOW, THREE, 2>(dblob, soff, toff, ntiles, state, sms, st);
    default: return cudaErrorInvalidValue;
    }
}

template <typename E>
int layouts_of(uint32_t gates, bool low)
{
    const uint32_t two = reg_mask<E, 0>() | reg_mask<E, 2>();
    const uint32_t three = two | reg_mask<E, 1>();
    if (gates & ~three) return 0;
    return (low || (gates & ~two)) ? 3 : 2;
}

}  // namespace

int span_tile_bits(int elem_bytes) { return elem_bytes == 8 ? SpanGeo<float2>::T : SpanGeo<double2>::T; }

// Register layouts a span pass runs through: 2 (A, B) when they hold every gate
// coordinate and the tile is not the low one, 3 (A, A', B) otherwise; 0 when the
// gates are not all on the layouts' register coordinates.
int span_layouts(int elem_bytes, uint32_t gates, bool low)
{
    if (elem_bytes == 8) {
        // complex64: the low pass always runs A -> A' -> B, a strided pass A -> B
        const int n = layouts_of<float2>(gates, low);
        return (n == 3 && !low) ? 0 : n;
    }
    return layouts_of<double2>(gates, low);
}

cudaError_t run_span(const uint8_t *dblob, uint64_t soff, uint64_t toff, uint64_t ntiles, int elem_bytes, bool low,
                     int layouts, int win, void *state, int sms, cudaStream_t st)
{
    if (elem_bytes == 8) {
        float2 *s = static_cast<float2 *>(state);
        if (low) return launch_span_win<float2, true, true>(dblob, soff, toff, ntiles, win, s, sms, st);
        if (layouts == 2) return launch_span_win<float2, false, false>(dblob, soff, toff, ntiles, win, s, sms, st);
        return cudaErrorInvalidValue;
    }
    double2 *s = static_cast<double2 *>(state);
    if (low) return launch_span_win<double2, true, true>(dblob, soff, toff, ntiles, win, s, sms, st);
    if (layouts == 3) return launch_span_win<double2, false, true>(dblob, soff, toff, ntiles, win, s, sms, st);
    return launch_span_win<double2, false, false>(dblob, soff, toff, ntiles, win, s, sms, st);
}

}  // namespace zxh
