// span.cu -- a U3 batch as span passes (sm_100a): up to 13 single-qubit gates per
// read-modify-write of the state, so a 30-qubit layer of U3 gates takes 3 passes
// (complex64 and complex128) instead of the reference's 30 sweeps
// (src/zxh/src/kernel/kernel_cuda.cu:390-423: one sweep per fused gate with a grid
// sync between) or the 5 (complex64) / 7 (complex128) register-row passes of
// u3pass.cu.
//
// A CTA (8 warps; two CTAs share an SM) works on tiles of 2^T amplitudes, 64 KiB:
// T = 13 for complex64 (32 amplitudes per thread in registers), T = 12 for
// complex128 (16 per thread). The tile's coordinates k = 0..T-1 are the real bits
// pos[k]: bits 0..c-1 (runs of 2^c contiguous amplitudes) and then the gates' bits;
// the other real bits enumerate tiles. A thread's amplitudes differ in R coordinates
// (its register coordinates), its lane and warp fix the other 5 + 3. The tile is
// read in layout A (a warp reads 2^min(c,5) contiguous amplitudes per segment) and
// written from a layout B; in between the amplitudes move between layouts through
// shared memory, and in each layout the gates on its register coordinates are
// register updates. Two forms:
//
// * Landing form (complex64). Layouts (register coordinates in register order):
//     A   regs 5, 6, 7, 8, 9     lanes 0..4        warps 10..12
//     A'  regs 0, 1, 2, 3, 9     lanes 4..8        warps 10..12
//     B   regs 4, 10, 11, 3, 12  lanes 0..2, 5, 6  warps 7..9
//     B2  regs 4, 10, 11, 12, 9  lanes 0..3, 5     warps 6..8
//   A strided pass whose gates A and B2 hold (c >= 4) runs A -> B2; the low pass
//   and strided passes with c = 3 run A -> A' -> B. Consecutive layouts share one
//   register coordinate, at the same register bit in both, so an exchange runs in
//   two rounds (that coordinate 0, then 1) through a 32 KiB half slab: each thread
//   writes half its registers and reads back the same half. The half slab's slot
//   of a tile index is a linear map chosen per exchange so that every write and
//   read is conflict-free. That leaves room for a 64 KiB landing slab per CTA: the
//   CTA's next tile lands there by 16-byte asynchronous copies while the current
//   one is worked on in registers (thread t copies the amplitude pairs at tile
//   indices 2t + 512k, k = 0..15, landing order = tile index).
//
// * Register form (complex128; complex64 behind a knob). Layouts:
//     complex64  (R = 5)                              complex128 (R = 4)
//     A   regs 5..9,  lanes 0..4,  warps 10..12        regs 5..8,  lanes 0..4,  warps 9..11
//     A'  regs 0..4,  lanes 5..9,  warps 10..12        regs 0..3,  lanes 4..8,  warps 9..11
//     B   regs 3, 4, 10..12, lanes 0..2, 5, 6,         regs 4, 9..11, lanes 0..2, 5, 6,
//         warps 7..9                                   warps 3, 7, 8
//   The tile is loaded straight into registers in A and the layouts change through
//   one 64 KiB XOR-swizzled slab. A pass runs A -> B when A and B hold all its gate
//   coordinates (complex64 strided passes, complex128 ones with c >= 4), else
//   A -> A' -> B.
//
// Gates are the real rotations of the planner's real split (U = e^{ia} P(b) R P(d),
// host.cpp): complex64 takes one paired FP32 FMA per amplitude and gate, complex128
// two FP64 FMAs; their phases ride in the windows. A window before the gates
// (prologue) is applied in A, one after them (epilogue) in the store layout: linear
// windows as one factor per thread times one per register pattern, others with
// in-tile quadratic terms by a Gray-code walk over the registers (32-bit turns for
// complex64, the full 64-bit turns for complex128).
#include "core.h"
#include "dev.cuh"
#include "host.h"
#include "sampler.h"

#include <algorithm>
#include <cuda_runtime.h>
#include <type_traits>

namespace zxh {

namespace {

constexpr int kSpanThreads = 256;  // 8 warps, two CTAs per SM (every form)

// Register form, complex64: 8-byte slab slots; a bank pair is slot bits 0..3: bits
// 0, 1, 2, 3 XOR bits 6, 7, 8, 5. In each layout the lanes of a warp access (its
// register index fixed) differ in 5 coordinates whose images span bits 0..3, so
// each access is the minimum two wavefronts.
struct GeoReg64 {
    using E = float2;
    static constexpr int T = 13, R = 5, W = 3;
    __host__ __device__ static constexpr int reg(int L, int r) { return L == 0 ? 5 + r : L == 1 ? r : (r < 2 ? 3 + r : T - 5 + r); }
    __host__ __device__ static constexpr int lane(int L, int b) { return L == 0 ? b : L == 1 ? 5 + b : (b < 3 ? b : 2 + b); }
    __host__ __device__ static constexpr int warp(int L, int w) { return L == 2 ? 7 + w : 10 + w; }
    __host__ __device__ static constexpr uint32_t slot(uint32_t t)
    {
        return t ^ ((t >> 6) & 1u) ^ (((t >> 7) & 1u) << 1) ^ (((t >> 8) & 1u) << 2) ^ (((t >> 5) & 1u) << 3);
    }
};

// Register form, complex128: 16-byte slots; a 16-byte access is served per 8
// consecutive lanes, whose slots must differ in bits 0..2: bits 0, 1, 2 XOR bits 4,
// 5, 6. Lane bits 0..2 are coordinates 0..2 (A, B) or 4..6 (A'), and with the other
// coordinate of each pair fixed the map is one-to-one.
struct GeoReg128 {
    using E = double2;
    static constexpr int T = 12, R = 4, W = 3;
    __host__ __device__ static constexpr int reg(int L, int r) { return L == 0 ? 5 + r : L == 1 ? r : (r == 0 ? 4 : 8 + r); }
    __host__ __device__ static constexpr int lane(int L, int b) { return L == 0 ? b : L == 1 ? 4 + b : (b < 3 ? b : 2 + b); }
    __host__ __device__ static constexpr int warp(int L, int w) { return L == 2 ? (w == 0 ? 3 : 6 + w) : 9 + w; }
    __host__ __device__ static constexpr uint32_t slot(uint32_t t) { return t ^ ((t >> 4) & 7u); }
};

// Landing form, complex64: layouts 0 A, 1 A', 2 B, 3 B2 (the table at the top);
// layout changes split on a shared register coordinate (HalfX).
struct GeoLand64 {
    using E = float2;
    static constexpr int T = 13, R = 5, W = 3;
    static constexpr int ACP = 2;  // amplitudes per 16-byte copy
    static constexpr bool EXP_SHARED = true;
    __host__ __device__ static constexpr int store_layout(bool three) { return three ? 2 : 3; }
    __host__ __device__ static constexpr int reg(int L, int r)
    {
        return L == 0 ? 5 + r
             : L == 1 ? (r < 4 ? r : 9)
             : L == 2 ? (r == 0 ? 4 : r == 3 ? 3 : r == 4 ? 12 : 9 + r)
                      : (r == 0 ? 4 : r == 4 ? 9 : 9 + r);
    }
    __host__ __device__ static constexpr int lane(int L, int b)
    {
        return L == 0 ? b : L == 1 ? 4 + b : L == 2 ? (b < 3 ? b : 2 + b) : (b < 4 ? b : 5);
    }
    __host__ __device__ static constexpr int warp(int L, int w) { return L < 2 ? 10 + w : L == 2 ? 7 + w : 6 + w; }
};

// Landing form, complex128: layouts 0 A, 1 A', 2 B (the table at the top); every
// pass runs A -> A' -> B. Four register coordinates per layout leave none to share,
// so a layout change splits on a warp coordinate both layouts have at the same
// warp bit (HalfW): coordinate 9 for A -> A', 7 for A' -> B. The exp table stays
// in global memory (read through L1) so that two CTAs fit an SM.
struct GeoLand128 {
    using E = double2;
    static constexpr int T = 12, R = 4, W = 3;
    static constexpr int ACP = 1;
    static constexpr bool EXP_SHARED = false;
    __host__ __device__ static constexpr int store_layout(bool) { return 2; }
    __host__ __device__ static constexpr int reg(int L, int r) { return L == 0 ? 5 + r : L == 1 ? r : (r == 0 ? 4 : 8 + r); }
    __host__ __device__ static constexpr int lane(int L, int b)
    {
        return L == 0 ? b : L == 1 ? (b < 3 ? 4 + b : 7 + b) : (b < 3 ? b : 2 + b);
    }
    __host__ __device__ static constexpr int warp(int L, int w) { return L == 0 ? 9 + w : w == 0 ? (L == 1 ? 9 : 3) : 6 + w; }
};

// The half-slab exchanges of the landing form: X = 1 A -> B2, 2 A -> A', 3 A' -> B.
// split: the shared register coordinate that picks the round; col(k): the half
// slab's slot bits of tile coordinate k (the slot of a tile index is the XOR of the
// columns of its set coordinates). Bank pair = slot bits 0..3; each map sends the
// lanes of a warp access, in both layouts, onto every bank pair twice.
// An 8-byte access is served per half warp, so lane bits 0..3 of each layout must
// map onto the 16 bank pairs (slot bits 0..3) one to one:
//   X = 1: the slot is the tile index with coordinate 9 taken out (lane bits 0..3
//          are coordinates 0..3 in A and in B2).
//   X = 2: the same, then slot bits 0..3 ^= coordinates 4..7 (lane bits 0..3 are
//          coordinates 0..3 in A, 4..7 in A').
//   X = 3: coordinate 3 taken out; slot bits 0..3 = coordinates 0 ^ 4, 1 ^ 6,
//          2 ^ 7, 5 (lane bits 0..3 are coordinates 4..7 in A', 0, 1, 2, 5 in B);
//          bits 4..11 = coordinates 4, 6, 7, 8, 9..12.
template <int X>
struct HalfX {
    static constexpr int split = X == 3 ? 3 : 9;
    __host__ __device__ static constexpr uint32_t col(int k)
    {
        if (X == 1) return k < 9 ? 1u << k : k == 9 ? 0u : 1u << (k - 1);
        if (X == 2) return (k >= 4 && k < 8) ? (1u << k) | (1u << (k - 4)) : k < 9 ? 1u << k : k == 9 ? 0u : 1u << (k - 1);
        switch (k) {
        case 0: return 1u;
        case 1: return 2u;
        case 2: return 4u;
        case 3: return 0u;
        case 4: return 1u | (1u << 4);
        case 5: return 1u << 3;
        case 6: return 2u | (1u << 5);
        case 7: return 4u | (1u << 6);
        default: return 1u << (k - 1);
        }
    }
    __host__ __device__ static constexpr uint32_t slot(uint32_t t)
    {
        uint32_t s = 0;
        for (int k = 0; k < 13; k++)
            if ((t >> k) & 1) s ^= col(k);
        return s;
    }
};

// The half-slab exchanges of the complex128 landing form (16-byte slots): the slot
// of a tile index is the index with the split coordinate taken out, its bits 0..2
// XOR bits 4..6. A 16-byte access is served per 8 consecutive lanes, whose lane
// bits 0..2 are coordinates 0..2 (A, B) or 4..6 (A'): one to one on slot bits 0..2.
template <int SPLIT, int WB>
struct HalfW {
    static constexpr int split = SPLIT, warp_bit = WB;
    __host__ __device__ static constexpr uint32_t slot(uint32_t t)
    {
        const uint32_t u = (t & ((1u << SPLIT) - 1u)) | ((t >> (SPLIT + 1)) << SPLIT);
        return u ^ ((u >> 4) & 7u);
    }
};

template <class G>
__host__ __device__ constexpr int span_nr() { return 1 << G::R; }  // amplitudes per thread

template <class G, int L>
__host__ __device__ constexpr uint32_t reg_index(int j)
{
    uint32_t t = 0;
    for (int r = 0; r < G::R; r++)
        if ((j >> r) & 1) t |= 1u << G::reg(L, r);
    return t;
}

template <class G, int L>
__host__ __device__ constexpr uint32_t reg_mask() { return reg_index<G, L>(span_nr<G>() - 1); }

template <class G, int L>
__host__ __device__ constexpr int reg_bit_of(int k)
{
    for (int r = 0; r < G::R; r++)
        if (G::reg(L, r) == k) return r;
    return -1;
}

template <class G, int L>
__device__ __forceinline__ uint32_t fixed_index(int lane, int warp)
{
    uint32_t t = 0;
#pragma unroll
    for (int b = 0; b < 5; b++) t |= uint32_t((lane >> b) & 1) << G::lane(L, b);
#pragma unroll
    for (int w = 0; w < G::W; w++) t |= uint32_t((warp >> w) & 1) << G::warp(L, w);
    return t;
}

// Real-address offset of tile index t.
template <class G>
__device__ __forceinline__ uint64_t real_of(uint32_t t, const uint8_t *pos)
{
    uint64_t o = 0;
#pragma unroll
    for (int k = 0; k < G::T; k++)
        if ((t >> k) & 1) o |= 1ULL << pos[k];
    return o;
}

// Register form: one exchange through the full slab. The slot map is linear over
// GF(2): slot(a | b) = slot(a) ^ slot(b) for disjoint a, b.
template <class G, int LA, int LB>
__device__ __forceinline__ void exchange(typename G::E (&x)[span_nr<G>()], typename G::E *slab, int lane, int warp)
{
    asm volatile("" : "+r"(lane), "+r"(warp));  // slot bases rebuilt here, not kept live across the tile loop
    const uint32_t sa = G::slot(fixed_index<G, LA>(lane, warp)), sb = G::slot(fixed_index<G, LB>(lane, warp));
    __syncthreads();  // the slab's previous reads are done
#pragma unroll
    for (int j = 0; j < span_nr<G>(); j++) slab[sa ^ G::slot(reg_index<G, LA>(j))] = x[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < span_nr<G>(); j++) x[j] = slab[sb ^ G::slot(reg_index<G, LB>(j))];
}

// Landing form: one exchange through the half slab, in two rounds on the shared
// register coordinate (register bit RS in both layouts): round h writes and reads
// back the registers whose bit RS is h.
template <class G, int LA, int LB, int X>
__device__ __forceinline__ void exchange_half(typename G::E (&x)[span_nr<G>()], typename G::E *slab, int lane, int warp)
{
    using H = HalfX<X>;
    constexpr int RS = reg_bit_of<G, LA>(H::split);
    static_assert(RS >= 0 && RS == reg_bit_of<G, LB>(H::split), "the split coordinate sits at one register bit");
    // the slot bases are rebuilt here from lane and warp (a few logic ops) rather
    // than kept live across the tile loop, where registers are short
    asm volatile("" : "+r"(lane), "+r"(warp));
    const uint32_t sa = H::slot(fixed_index<G, LA>(lane, warp)), sb = H::slot(fixed_index<G, LB>(lane, warp));
#pragma unroll
    for (int h = 0; h < 2; h++) {
        __syncthreads();  // the half slab's previous reads are done
#pragma unroll
        for (int j = 0; j < span_nr<G>(); j++)
            if (((j >> RS) & 1) == h) slab[sa ^ H::slot(reg_index<G, LA>(j))] = x[j];
        __syncthreads();
#pragma unroll
        for (int j = 0; j < span_nr<G>(); j++)
            if (((j >> RS) & 1) == h) x[j] = slab[sb ^ H::slot(reg_index<G, LB>(j))];
    }
}

// Landing form, complex128: one exchange through the half slab, in two rounds on
// the shared warp coordinate: round h moves the tile entries of the warps whose
// warp bit WB is h (the others wait at the barriers).
template <class G, int LA, int LB, class H>
__device__ __forceinline__ void exchange_warps(typename G::E (&x)[span_nr<G>()], typename G::E *slab, int lane, int warp)
{
    static_assert(G::warp(LA, H::warp_bit) == H::split && G::warp(LB, H::warp_bit) == H::split,
                  "the split coordinate is the same warp bit in both layouts");
    asm volatile("" : "+r"(lane), "+r"(warp));  // slot bases rebuilt here, not kept live across the tile loop
    const uint32_t sa = H::slot(fixed_index<G, LA>(lane, warp)), sb = H::slot(fixed_index<G, LB>(lane, warp));
    const bool mine = (warp >> H::warp_bit) & 1;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        __syncthreads();  // the half slab's previous reads are done
        if (int(mine) == h) {
#pragma unroll
            for (int j = 0; j < span_nr<G>(); j++) slab[sa ^ H::slot(reg_index<G, LA>(j))] = x[j];
        }
        __syncthreads();
        if (int(mine) == h) {
#pragma unroll
            for (int j = 0; j < span_nr<G>(); j++) x[j] = slab[sb ^ H::slot(reg_index<G, LB>(j))];
        }
    }
}

// The rotations of layout L's register coordinates that are in `mask`, each with
// one coefficient factored out (SpanDev): rot[k] = (tau, 0): x' = x - tau y,
// y' = y + tau x; (mu, 1): x' = mu x - y, y' = x + mu y.
template <class G, int L>
__device__ __forceinline__ void rotate(typename G::E (&x)[span_nr<G>()], const typename G::E *rot, uint32_t mask)
{
    using E = typename G::E;
    constexpr int NR = span_nr<G>();
#pragma unroll
    for (int r = 0; r < G::R; r++) {
        const int k = G::reg(L, r);
        if (!((mask >> k) & 1)) continue;
        const E cm = rot[k];
        if constexpr (std::is_same_v<E, float2>) {
            const float2 q = make_float2(cm.x, cm.x);
            if (cm.y == 0.0f) {
                const float2 nq = make_float2(-cm.x, -cm.x);
#pragma unroll
                for (int j = 0; j < NR; j++) {
                    if ((j >> r) & 1) continue;
                    const float2 lo = x[j], hi = x[j | (1 << r)];
                    x[j] = __ffma2_rn(nq, hi, lo);
                    x[j | (1 << r)] = __ffma2_rn(q, lo, hi);
                }
            } else {
#pragma unroll
                for (int j = 0; j < NR; j++) {
                    if ((j >> r) & 1) continue;
                    const float2 lo = x[j], hi = x[j | (1 << r)];
                    x[j] = __ffma2_rn(q, lo, make_float2(-hi.x, -hi.y));
                    x[j | (1 << r)] = __ffma2_rn(q, hi, lo);
                }
            }
        } else {
            const double q = cm.x;
            if (cm.y == 0.0) {
#pragma unroll
                for (int j = 0; j < NR; j++) {
                    if ((j >> r) & 1) continue;
                    const double2 lo = x[j], hi = x[j | (1 << r)];
                    x[j] = make_double2(fma(-q, hi.x, lo.x), fma(-q, hi.y, lo.y));
                    x[j | (1 << r)] = make_double2(fma(q, lo.x, hi.x), fma(q, lo.y, hi.y));
                }
            } else {
#pragma unroll
                for (int j = 0; j < NR; j++) {
                    if ((j >> r) & 1) continue;
                    const double2 lo = x[j], hi = x[j | (1 << r)];
                    x[j] = make_double2(fma(q, lo.x, -hi.x), fma(q, lo.y, -hi.y));
                    x[j | (1 << r)] = make_double2(fma(q, hi.x, lo.x), fma(q, hi.y, lo.y));
                }
            }
        }
    }
}

// A window's phase at a thread's amplitudes in layout L for one tile, in a form
// that needs few registers while the amplitudes are live: linear windows give
// one factor per thread (times rowf[j] per register pattern); others give the
// thread's constant and its R register coefficients in turns (32-bit turns for
// complex64, 64-bit for complex128), the register x register terms a factor
// rowf[j] per register pattern.
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

template <class G, int L, bool LINEAR>
__device__ __forceinline__ SpanWin<typename G::E> span_window_setup(const uint8_t *blob, const DiagDev &dd,
                                                                    const typename G::E *s_exp, uint64_t base,
                                                                    int lane, int warp, int64_t fixc)
{
    SpanWin<typename G::E> sw;
    if constexpr (LINEAR) {
        // only linear terms: the tile's out-of-tile bits give one sum shared by all
        // threads, the thread's lane and warp coordinates a constant (fixc)
        const LinTerm *ol = reinterpret_cast<const LinTerm *>(blob + dd.off_out_lin);
        if constexpr (std::is_same_v<typename G::E, float2>) {
            // complex64: the sum in 32-bit turns (each term rounded once), one warp
            // reduction instruction instead of a shuffle tree of 64-bit values
            uint32_t K = 0;
            for (uint32_t q = uint32_t(lane); q < dd.n_out_lin; q += 32)
                if ((base >> ol[q].bit) & 1) K += turns32(ol[q].coef);
            sw.f = phase_factor32(s_exp, __reduce_add_sync(0xffffffffu, K) + turns32(dd.c0 + fixc));
        } else {
            int64_t K = 0;
            for (uint32_t q = uint32_t(lane); q < dd.n_out_lin; q += 32)
                if ((base >> ol[q].bit) & 1) K += ol[q].coef;
            sw.f = phase_factor(s_exp, warp_sum_i64(K) + dd.c0 + fixc);
        }
        return sw;
    }
    constexpr uint32_t RM = reg_mask<G, L>();
    const uint32_t fix = fixed_index<G, L>(lane, warp);
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
    int64_t w[G::R];
#pragma unroll
    for (int r = 0; r < G::R; r++) w[r] = __shfl_sync(0xffffffffu, da, G::reg(L, r));
    // in-tile quadratic terms with a fixed coordinate set
    const QuadTerm *iq = reinterpret_cast<const QuadTerm *>(blob + dd.off_in_quad);
    for (uint32_t q = 0; q < dd.n_in_quad; q++) {
        const QuadTerm t = iq[q];
        const bool ri = (RM >> t.i) & 1, rj = (RM >> t.j) & 1;
        if (ri && rj) continue;  // register x register: in rowf
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

template <class G, bool LINEAR>
__device__ __forceinline__ void span_window_apply(typename G::E (&x)[span_nr<G>()], const SpanWin<typename G::E> &sw,
                                                  const typename G::E *rowf, bool quad_regs,
                                                  const typename G::E *s_exp)
{
    using E = typename G::E;
    if constexpr (LINEAR) {
        // a linear phase factors over the register bits: rowf[jl + 4 jh] = rowf[jl]
        // rowf[4 jh], so four per-thread factors and one table load per four patterns
        E lo[4];
#pragma unroll
        for (int jl = 0; jl < 4; jl++) lo[jl] = cmul(sw.f, rowf[jl]);
#pragma unroll
        for (int jh = 0; jh < span_nr<G>() / 4; jh++) {
            const E hf = rowf[jh << 2];
#pragma unroll
            for (int jl = 0; jl < 4; jl++) {
                const int j = jl | (jh << 2);
                x[j] = cmul(x[j], jh ? cmul(lo[jl], hf) : lo[jl]);
            }
        }
    } else {
        // the phase of pattern j = jl + 4 jh is a + w0 jl0 + w1 jl1 + sum_r>=2 w_r jh_r-2
        // (+ the register x register terms): four factors for jl, one per jh, and
        // their product per amplitude (each factor evaluated from turns, so no
        // product chains more than three factors)
        E lo[4];
#pragma unroll
        for (int jl = 0; jl < 4; jl++) lo[jl] = span_phase(s_exp, sw.a + ((jl & 1) ? sw.w[0] : 0) + ((jl & 2) ? sw.w[1] : 0));
#pragma unroll
        for (int jh = 0; jh < span_nr<G>() / 4; jh++) {
            decltype(sw.a) t = 0;
#pragma unroll
            for (int r = 2; r < G::R; r++)
                if ((jh >> (r - 2)) & 1) t += sw.w[r];
            const E hf = span_phase(s_exp, t);
#pragma unroll
            for (int jl = 0; jl < 4; jl++) {
                const int j = jl | (jh << 2);
                E f = cmul(lo[jl], hf);
                if (quad_regs) f = cmul(f, rowf[j]);
                x[j] = cmul(x[j], f);
            }
        }
    }
}

// Per-CTA tables of a span pass, filled once per launch by span_setup; LS is the
// store layout.
template <class G, int WIN, bool EXPS = true>
struct SpanShared {
    using E = typename G::E;
    E exp[(WIN && EXPS) ? (1 << kExpTableBits) : 1];  // WIN != 0 and the table in shared memory
    const E *gtab;                                    // else the blob's copy (read through L1)
    // the exp table: a shared-memory address the compiler can see, or the global copy
    __device__ __forceinline__ const E *table() const
    {
        if constexpr (EXPS) return exp;
        else return gtab;
    }
    E rot[kSpanBits];                       // (coefficient, form) per coordinate
    uint64_t roff[2][span_nr<G>()];         // real offsets of the register patterns: layout A (loads), LS (stores)
    uint64_t soff[G::R];                    // real offset of each register coordinate of LS
    E rowf[2][span_nr<G>()];                // window 0 in layout A, 1 in LS: linear windows the
                                            // pattern's factor, others its register x register factor
    int quad_regs[2];                       // window d has register x register terms
    uint64_t grp[16];                       // landing form: real offset of tile index k << 9
    int64_t fixl[2][32], fixw[2][8];        // linear windows: lin_in summed over a thread's lane / warp coordinates
    uint8_t pos[16];
};

template <class G, int LS, int WIN, bool EXPS>
__device__ __forceinline__ void span_setup(SpanShared<G, WIN, EXPS> &sh, const SpanDev &p, const uint8_t *blob,
                                           uint64_t toff, int tid)
{
    using E = typename G::E;
    constexpr int NR = span_nr<G>();
    if (tid < 16) sh.pos[tid] = p.pos[tid];
    if (tid < 2) sh.quad_regs[tid] = 0;
    if (tid < G::T) {
        sh.rot[tid].x = decltype(E{}.x)(p.rot[tid][0]);
        sh.rot[tid].y = decltype(E{}.x)(p.rot[tid][1]);
    }
    if constexpr (WIN != 0) {
        const E *tab = reinterpret_cast<const E *>(blob + toff);
        if constexpr (EXPS) {
            for (int i = tid; i < (1 << kExpTableBits); i += kSpanThreads) sh.exp[i] = tab[i];
        } else {
            if (tid == 0) sh.gtab = tab;
        }
    }
    __syncthreads();
    if (tid < 2 * NR) {
        const int L = tid / NR, j = tid % NR;
        sh.roff[L][j] = real_of<G>(L ? reg_index<G, LS>(j) : reg_index<G, 0>(j), sh.pos);
        if (L && j < G::R) sh.soff[j] = 1ULL << sh.pos[G::reg(LS, j)];
    }
    if (WIN && tid >= 2 * NR && tid < 4 * NR) {
        // tile-independent window parts: the per-pattern factors of linear windows,
        // the register x register quadratic terms of the others
        const int d = (tid - 2 * NR) / NR, j = tid % NR;
        const uint64_t ow = d ? p.off_post : p.off_pre;
        int64_t qa = 0, lb = 0;
        if (ow) {
            const DiagDev &dd = *reinterpret_cast<const DiagDev *>(blob + ow);
            const uint32_t t = d ? reg_index<G, LS>(j) : reg_index<G, 0>(j);
            const QuadTerm *iq = reinterpret_cast<const QuadTerm *>(blob + dd.off_in_quad);
            for (uint32_t q = 0; q < dd.n_in_quad; q++)
                if (((t >> iq[q].i) & 1) && ((t >> iq[q].j) & 1)) qa += iq[q].coef;
            for (int k = 0; k < G::T; k++)
                if ((t >> k) & 1) lb += dd.lin_in[k];
        }
        sh.rowf[d][j] = phase_factor(sh.table(), WIN == 1 ? lb : qa);
        if (qa != 0) sh.quad_regs[d] = 1;
    }
    // landing form: tile index of a thread's k-th 16-byte copy = (tid + 256 k) x amplitudes per copy
    if (tid >= 4 * NR && tid < 4 * NR + 16) {
        constexpr uint32_t acp = 16 / sizeof(E);
        sh.grp[tid - 4 * NR] = real_of<G>(uint32_t(tid - 4 * NR) * 256u * acp, sh.pos);
    }
    if (WIN == 1 && tid >= 160 && tid < 240) {
        // window d's coefficients summed over lane bits (fixl) and warp bits (fixw)
        const int i = tid - 160, d = i / 40, v = i % 40;
        const uint64_t ow = d ? p.off_post : p.off_pre;
        int64_t c = 0;
        if (ow) {
            const DiagDev &dd = *reinterpret_cast<const DiagDev *>(blob + ow);
            const int L = d ? LS : 0;
            if (v < 32) {
                for (int b = 0; b < 5; b++)
                    if ((v >> b) & 1) c += dd.lin_in[L == 0 ? G::lane(0, b) : G::lane(LS, b)];
            } else {
                for (int w = 0; w < G::W; w++)
                    if (((v - 32) >> w) & 1) c += dd.lin_in[L == 0 ? G::warp(0, w) : G::warp(LS, w)];
            }
        }
        if (v < 32) sh.fixl[d][v] = c;
        else sh.fixw[d][v - 32] = c;
    }
    __syncthreads();
}

// First real address of a tile: the strided passes insert zeros at the tile's real
// bits (ascending); the low pass's tiles are contiguous.
template <class G, bool LOW>
__device__ __forceinline__ uint64_t span_tile_base(uint64_t tile, const uint8_t *pos)
{
    if constexpr (LOW) return tile << G::T;
#pragma unroll
    for (int k = 0; k < G::T; k++) {
        const uint32_t b = pos[k];
        tile = ((tile >> b) << (b + 1)) | (tile & ((1ULL << b) - 1ULL));
    }
    return tile;
}

// The gates of each layout (A, A', the store layout LS) and where the rotations'
// common factor goes: into a linear window's per-thread factor where there is one,
// else one multiply before the store.
template <typename E>
struct SpanGates {
    uint32_t gA, gAp, gB;
    decltype(E{}.x) scale;
    bool scale_pre, scale_post, scale_end;
};

template <class G, bool THREE, int LS, int WIN>
__device__ __forceinline__ SpanGates<typename G::E> span_gates(const SpanDev &p)
{
    SpanGates<typename G::E> g;
    const uint32_t gm = p.gates;
    g.gA = gm & reg_mask<G, 0>();
    g.gAp = THREE ? (gm & reg_mask<G, 1>() & ~g.gA) : 0u;
    g.gB = gm & reg_mask<G, LS>() & ~g.gA & ~g.gAp;
    g.scale = decltype(g.scale)(p.scale);
    g.scale_pre = WIN == 1 && p.off_pre != 0;
    g.scale_post = WIN == 1 && !g.scale_pre && p.off_post != 0;
    g.scale_end = !g.scale_pre && !g.scale_post;
    return g;
}

__device__ __forceinline__ void span_scale(float2 &x, float s) { x = __fmul2_rn(make_float2(s, s), x); }
__device__ __forceinline__ void span_scale(double2 &x, double s) { x = make_double2(x.x * s, x.y * s); }

template <class G, int LS, int WIN, bool EXPS>
__device__ __forceinline__ void span_windows_setup(SpanWin<typename G::E> &wpre, SpanWin<typename G::E> &wpost,
                                                   const SpanDev &p, const uint8_t *blob,
                                                   const SpanShared<G, WIN, EXPS> &sh,
                                                   const SpanGates<typename G::E> &g, uint64_t base, int lane, int warp)
{
    if constexpr (WIN != 0) {
        if (p.off_pre) {
            wpre = span_window_setup<G, 0, WIN == 1>(blob, *reinterpret_cast<const DiagDev *>(blob + p.off_pre), sh.table(),
                                                     base, lane, warp, sh.fixl[0][lane] + sh.fixw[0][warp]);
            if (g.scale_pre) span_scale(wpre.f, g.scale);
        }
        if (p.off_post) {
            wpost = span_window_setup<G, LS, WIN == 1>(blob, *reinterpret_cast<const DiagDev *>(blob + p.off_post),
                                                       sh.table(), base, lane, warp, sh.fixl[1][lane] + sh.fixw[1][warp]);
            if (g.scale_post) span_scale(wpost.f, g.scale);
        }
    }
}

// WIN: 0 no window, 1 windows with linear terms only, 2 any windows (quadratic
// terms; no multi-bit selectors). LOW: the tile is real bits 0..T-1. THREE: the
// layouts A, A', B (else A and B, or A and B2 in the landing form).
//
// Register form: each CTA works on one tile at a time: the windows' per-tile parts
// computed before the loads (few registers stay live across the tile), loads in
// layout A straight into registers, exchanges through the slab, stores from B.
template <class G, bool LOW, bool THREE, int WIN>
__global__ void __launch_bounds__(kSpanThreads, 2) span_kernel(const uint8_t *__restrict__ blob, uint64_t soff,
                                                              uint64_t toff, typename G::E *__restrict__ state)
{
    using E = typename G::E;
    constexpr int NR = span_nr<G>();
    extern __shared__ __align__(128) unsigned char s_raw[];
    E *slab = reinterpret_cast<E *>(s_raw);  // 2^T slots
    __shared__ SpanShared<G, WIN> sh;

    const SpanDev &p = *reinterpret_cast<const SpanDev *>(blob + soff);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    span_setup<G, 2>(sh, p, blob, toff, tid);

    const uint64_t offA = real_of<G>(fixed_index<G, 0>(lane, warp), sh.pos);
    const uint64_t offB = real_of<G>(fixed_index<G, 2>(lane, warp), sh.pos);
    const SpanGates<E> g = span_gates<G, THREE, 2, WIN>(p);
    const uint64_t ntiles = p.ntiles;

    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t base = span_tile_base<G, LOW>(tile, sh.pos);
        [[maybe_unused]] SpanWin<E> wpre, wpost;
        span_windows_setup<G, 2, WIN, true>(wpre, wpost, p, blob, sh, g, base, lane, warp);
        E x[NR];
        const E *src = state + base + offA;
#pragma unroll
        for (int j = 0; j < NR; j++) x[j] = __ldcs(src + sh.roff[0][j]);
        if constexpr (WIN != 0) {
            if (p.off_pre) span_window_apply<G, WIN == 1>(x, wpre, sh.rowf[0], sh.quad_regs[0] != 0, sh.table());
        }
        rotate<G, 0>(x, sh.rot, g.gA);
        if constexpr (THREE) {
            exchange<G, 0, 1>(x, slab, lane, warp);
            rotate<G, 1>(x, sh.rot, g.gAp);
            exchange<G, 1, 2>(x, slab, lane, warp);
        } else {
            exchange<G, 0, 2>(x, slab, lane, warp);
        }
        rotate<G, 2>(x, sh.rot, g.gB);
        if constexpr (WIN != 0) {
            if (p.off_post) span_window_apply<G, WIN == 1>(x, wpost, sh.rowf[1], sh.quad_regs[1] != 0, sh.table());
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

// A pass's rotation coefficients and tile coordinates as a kernel parameter: read
// from the constant bank where a gate is applied or a tile's base address is formed,
// with no shared-memory load.
template <typename E>
struct SpanConst {
    E r[kSpanBits];
    uint8_t pos[16];
};

// Landing form: the dynamic shared memory holds the landing slab (2^T slots) and
// the half slab (2^(T-1) slots). A tile's turn: wait for its copies, read it from
// the landing slab in layout A, then (once every thread has read it) start the
// copies of the CTA's next tile into the landing slab, and work on this one.
template <class G, bool LOW, bool THREE, int WIN>
__global__ void __launch_bounds__(kSpanThreads, 2)
    span_land_kernel(const uint8_t *__restrict__ blob, uint64_t soff, uint64_t toff, typename G::E *__restrict__ state,
                     const __grid_constant__ SpanConst<typename G::E> kc)
{
    using E = typename G::E;
    constexpr int NR = span_nr<G>();
    constexpr int LS = G::store_layout(THREE);  // B, or B2 for two-layout complex64 passes
    constexpr bool EXPS = G::EXP_SHARED;
    static_assert(THREE || std::is_same_v<G, GeoLand64>, "complex128 landing passes run A -> A' -> B");
    extern __shared__ __align__(128) unsigned char s_raw[];
    E *s_land = reinterpret_cast<E *>(s_raw);
    E *half = s_land + (1 << G::T);
    __shared__ SpanShared<G, WIN, EXPS> sh;

    const SpanDev &p = *reinterpret_cast<const SpanDev *>(blob + soff);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    span_setup<G, LS>(sh, p, blob, toff, tid);

    // per-thread offsets kept in shared memory (registers are the scarce resource):
    // this thread's first 16-byte copy in each group of 256 x ACP tile indices, and
    // its store pattern's base
    __shared__ uint64_t s_cpo[kSpanThreads], s_offS[kSpanThreads];
    s_cpo[tid] = real_of<G>(uint32_t(tid) * G::ACP, sh.pos);
    s_offS[tid] = real_of<G>(fixed_index<G, LS>(lane, warp), sh.pos);
    const uint32_t fa = fixed_index<G, 0>(lane, warp);
    const SpanGates<E> g = span_gates<G, THREE, LS, WIN>(p);
    const uint64_t ntiles = p.ntiles;

    // the copies of a tile into the landing slab; a group is committed either way
    auto issue = [&](uint64_t tile) {
        if (tile < ntiles) {
            // copy k's source by a Gray-code walk over k from the offsets of its four bits
            const E *src = state + span_tile_base<G, LOW>(tile, kc.pos) + s_cpo[tid];
            const uint64_t go[4] = {sh.grp[1], sh.grp[2], sh.grp[4], sh.grp[8]};
#pragma unroll
            for (int kk = 0; kk < 16; kk++) {
                const int k = kk ^ (kk >> 1);
                if (kk > 0) {
                    const int fb = ctz_const(kk);
                    if ((k >> fb) & 1) src += go[fb];
                    else src -= go[fb];
                }
                cp_async16(s_land + (tid + 256 * k) * G::ACP, src);
            }
        }
        cp_async_commit();
    };
    issue(blockIdx.x);

    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t base = span_tile_base<G, LOW>(tile, kc.pos);
        [[maybe_unused]] SpanWin<E> wpre, wpost;
        span_windows_setup<G, LS>(wpre, wpost, p, blob, sh, g, base, lane, warp);
        cp_async_wait<0>();  // this thread's copies of the tile have landed
        __syncthreads();     // and everyone's
        E x[NR];
#pragma unroll
        for (int j = 0; j < NR; j++) x[j] = s_land[fa | reg_index<G, 0>(j)];
        __syncthreads();  // every thread has read the landing slab
        issue(tile + gridDim.x);
        if constexpr (WIN != 0) {
            if (p.off_pre) span_window_apply<G, WIN == 1>(x, wpre, sh.rowf[0], sh.quad_regs[0] != 0, sh.table());
        }
        rotate<G, 0>(x, kc.r, g.gA);
        if constexpr (std::is_same_v<G, GeoLand64>) {
            if constexpr (THREE) {
                exchange_half<G, 0, 1, 2>(x, half, lane, warp);
                rotate<G, 1>(x, kc.r, g.gAp);
                exchange_half<G, 1, 2, 3>(x, half, lane, warp);
            } else {
                exchange_half<G, 0, 3, 1>(x, half, lane, warp);
            }
        } else {
            exchange_warps<G, 0, 1, HalfW<9, 0>>(x, half, lane, warp);
            rotate<G, 1>(x, kc.r, g.gAp);
            exchange_warps<G, 1, 2, HalfW<7, 1>>(x, half, lane, warp);
        }
        rotate<G, LS>(x, kc.r, g.gB);
        if constexpr (WIN != 0) {
            if (p.off_post) span_window_apply<G, WIN == 1>(x, wpost, sh.rowf[1], sh.quad_regs[1] != 0, sh.table());
        }
        if (g.scale_end) {
#pragma unroll
            for (int j = 0; j < NR; j++) span_scale(x[j], g.scale);
        }
        // the store patterns walked in Gray-code order: one 64-bit add per amplitude
        // from the register coordinates' offsets, instead of a table load each
        E *dst = state + base + s_offS[tid];
        uint64_t so[G::R];
#pragma unroll
        for (int r = 0; r < G::R; r++) so[r] = sh.soff[r];
#pragma unroll
        for (int jj = 0; jj < NR; jj++) {
            const int gj = jj ^ (jj >> 1);
            if (jj > 0) {
                const int fb = ctz_const(jj);
                if ((gj >> fb) & 1) dst += so[fb];
                else dst -= so[fb];
            }
            __stcs(dst, x[gj]);
        }
    }
    cp_async_wait<0>();  // the last committed group is empty; nothing lands after exit
}

// grid: every resident CTA, at most one per tile
template <class K>
unsigned span_grid(K kern, size_t smem, uint64_t ntiles, int sms)
{
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSpanThreads, smem);
    if (per_sm < 1) per_sm = 1;
    return unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(sms) * uint64_t(per_sm))));
}

template <class G, bool LOW, bool THREE, int WIN>
cudaError_t launch_span(const uint8_t *dblob, uint64_t soff, uint64_t toff, uint64_t ntiles, void *state, int sms,
                        cudaStream_t st)
{
    using E = typename G::E;
    auto kern = span_kernel<G, LOW, THREE, WIN>;
    const size_t smem = sizeof(E) << G::T;  // 64 KiB
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    kern<<<span_grid(kern, smem, ntiles, sms), kSpanThreads, smem, st>>>(dblob, soff, toff, static_cast<E *>(state));
    return cudaGetLastError();
}

template <class G, bool LOW, bool THREE, int WIN>
cudaError_t launch_span_land(const uint8_t *dblob, uint64_t soff, uint64_t toff, uint64_t ntiles, void *state,
                             const double (*rot)[2], const uint8_t *pos, int sms, cudaStream_t st)
{
    using E = typename G::E;
    SpanConst<E> kc;
    for (int k = 0; k < kSpanBits; k++) {
        kc.r[k].x = decltype(E{}.x)(rot[k][0]);
        kc.r[k].y = decltype(E{}.x)(rot[k][1]);
    }
    for (int k = 0; k < 16; k++) kc.pos[k] = pos[k];
    auto kern = span_land_kernel<G, LOW, THREE, WIN>;
    const size_t smem = (sizeof(E) << G::T) + (sizeof(E) << (G::T - 1));  // 64 + 32 KiB
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    kern<<<span_grid(kern, smem, ntiles, sms), kSpanThreads, smem, st>>>(dblob, soff, toff, static_cast<E *>(state),
                                                                         kc);
    return cudaGetLastError();
}

template <int FORM, bool LOW, bool THREE>
cudaError_t launch_span_win(const uint8_t *dblob, uint64_t soff, uint64_t toff, uint64_t ntiles, int win, void *state,
                            const double (*rot)[2], const uint8_t *pos, int sms, cudaStream_t st)
{
    // FORM: 0 register form complex64, 1 register form complex128, 2 landing form
    // complex64, 3 landing form complex128
    auto go = [&](auto w) -> cudaError_t {
        constexpr int W = decltype(w)::value;
        if constexpr (FORM == 0) return launch_span<GeoReg64, LOW, THREE, W>(dblob, soff, toff, ntiles, state, sms, st);
        else if constexpr (FORM == 1)
            return launch_span<GeoReg128, LOW, THREE, W>(dblob, soff, toff, ntiles, state, sms, st);
        else if constexpr (FORM == 2)
            return launch_span_land<GeoLand64, LOW, THREE, W>(dblob, soff, toff, ntiles, state, rot, pos, sms, st);
        else return launch_span_land<GeoLand128, LOW, THREE, W>(dblob, soff, toff, ntiles, state, rot, pos, sms, st);
    };
    switch (win) {
    case 0: return go(std::integral_constant<int, 0>{});
    case 1: return go(std::integral_constant<int, 1>{});
    case 2: return go(std::integral_constant<int, 2>{});
    default: return cudaErrorInvalidValue;
    }
}

// 2 layouts when the first and the store layout hold every gate coordinate and the
// tile is not the low one, 3 when A' is needed too, 0 when no layout holds some gate
template <class G, int L2>
int layouts_of(uint32_t gates, bool low)
{
    const uint32_t two = reg_mask<G, 0>() | reg_mask<G, L2>();
    const uint32_t three = reg_mask<G, 0>() | reg_mask<G, 1>() | reg_mask<G, 2>();
    if (low || (gates & ~two)) return (gates & ~three) ? 0 : 3;
    return 2;
}

}  // namespace

int span_tile_bits(int elem_bytes) { return elem_bytes == 8 ? GeoReg64::T : GeoReg128::T; }

int span_layouts(int elem_bytes, uint32_t gates, bool low, bool land)
{
    if (elem_bytes != 8) {
        const int n = layouts_of<GeoReg128, 2>(gates, low);
        return (land && n) ? 3 : n;  // the complex128 landing form always runs A -> A' -> B
    }
    if (land) return layouts_of<GeoLand64, 3>(gates, low);
    // complex64 register form: the low pass runs A -> A' -> B, a strided pass A -> B
    const int n = layouts_of<GeoReg64, 2>(gates, low);
    return (n == 3 && !low) ? 0 : n;
}

cudaError_t run_span(const uint8_t *dblob, uint64_t soff, uint64_t toff, uint64_t ntiles, int elem_bytes, bool low,
                     int layouts, bool land, int win, void *state, const double (*rot)[2], const uint8_t *pos, int sms,
                     cudaStream_t st)
{
    if (layouts != 2 && layouts != 3) return cudaErrorInvalidValue;
    const bool three = layouts == 3;
    if (elem_bytes == 16) {
        if (land) {
            if (!three) return cudaErrorInvalidValue;
            return low ? launch_span_win<3, true, true>(dblob, soff, toff, ntiles, win, state, rot, pos, sms, st)
                       : launch_span_win<3, false, true>(dblob, soff, toff, ntiles, win, state, rot, pos, sms, st);
        }
        if (low) return launch_span_win<1, true, true>(dblob, soff, toff, ntiles, win, state, rot, pos, sms, st);
        return three ? launch_span_win<1, false, true>(dblob, soff, toff, ntiles, win, state, rot, pos, sms, st)
                     : launch_span_win<1, false, false>(dblob, soff, toff, ntiles, win, state, rot, pos, sms, st);
    }
    if (land) {
        if (low) return launch_span_win<2, true, true>(dblob, soff, toff, ntiles, win, state, rot, pos, sms, st);
        return three ? launch_span_win<2, false, true>(dblob, soff, toff, ntiles, win, state, rot, pos, sms, st)
                     : launch_span_win<2, false, false>(dblob, soff, toff, ntiles, win, state, rot, pos, sms, st);
    }
    if (low) return launch_span_win<0, true, true>(dblob, soff, toff, ntiles, win, state, rot, pos, sms, st);
    if (three) return cudaErrorInvalidValue;
    return launch_span_win<0, false, false>(dblob, soff, toff, ntiles, win, state, rot, pos, sms, st);
}

}  // namespace zxh
