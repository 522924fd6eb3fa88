// span.cu -- a U3 batch as span passes (sm_100a, complex64): up to 12 single-qubit
// gates per read-modify-write of the state, so a 30-qubit layer of U3 gates takes 3
// passes instead of the reference's 30 sweeps (src/zxh/src/kernel/kernel_cuda.cu:
// 390-423: one sweep per fused gate with a grid sync between) or the 5 of the
// register-row passes (u3pass.cu).
//
// A CTA (4 warps; four CTAs share an SM) owns a tile of 2^12 amplitudes, 32 per
// thread in registers. The tile's coordinates k = 0..11 are the real bits pos[k]:
// bits 0..c-1 (runs of 2^c contiguous amplitudes) and then the gates' bits; the
// other real bits enumerate tiles. A thread's 32 amplitudes differ in 5
// coordinates (its register bits), its lane and warp fix the other 7. Layouts:
//   A   registers on coordinates 5..9,        lanes 0..4,          warps 10, 11
//   A'  registers on coordinates 0..4,        lanes 5..9,          warps 10, 11
//   B   registers on coordinates 3, 4, 9..11, lanes 0, 1, 2, 5, 6, warps 7, 8
// The tile is loaded in A (a warp reads 2^min(c,5) contiguous amplitudes per
// segment), and the amplitudes move between layouts through one 32 KiB shared
// slab (XOR-swizzled, so every write and read of a layout change is conflict-free).
// In each layout the gates on its register coordinates are register updates. A
// strided pass (c >= 3: 12 - c gates on high bits) runs A -> B; the low pass (the
// tile is bits 0..11) runs A -> A' -> B. The tile is written from B.
//
// Gates are the real rotations of the planner's real split (U = e^{ia} P(b) R P(d),
// host.cpp): two paired FP32 FMAs per amplitude and gate; their phases ride in the
// windows. A window before the gates (prologue) is applied in A, one after them
// (epilogue) in B: linear windows as one factor per thread times one per register
// pattern, others with in-tile quadratic terms by a Gray-code walk over the
// registers in 32-bit turns.
#include "core.h"
#include "dev.cuh"
#include "host.h"
#include "sampler.h"

#include <algorithm>
#include <cuda_runtime.h>

namespace zxh {

namespace {

constexpr int kT = kSpanBits;                                    // 13 tile coordinates
constexpr int kR = 5;                                            // register coordinates per layout
constexpr int kNR = 1 << kR;                                     // amplitudes per thread
constexpr int kSW = kT - 10;                                     // warp coordinates: 3
constexpr int kSpanThreads = 32 << kSW;                          // 8 warps, two CTAs per SM
constexpr uint32_t kTileBytes = uint32_t(sizeof(float2)) << kT;  // 64 KiB

// Register, lane and warp coordinates of each layout (A, A', B).
__host__ __device__ constexpr int reg_coord(int L, int r)
{
    return L == 0 ? 5 + r : L == 1 ? r : (r < 2 ? 3 + r : kT - 5 + r);
}
__host__ __device__ constexpr int lane_coord(int L, int b) { return L == 0 ? b : L == 1 ? 5 + b : (b < 3 ? b : 2 + b); }
__host__ __device__ constexpr int warp_coord(int L, int w) { return L == 2 ? 7 + w : 10 + w; }

template <int L>
__host__ __device__ constexpr uint32_t reg_index(int j)
{
    uint32_t t = 0;
    for (int r = 0; r < kR; r++)
        if ((j >> r) & 1) t |= 1u << reg_coord(L, r);
    return t;
}

template <int L>
__host__ __device__ constexpr uint32_t reg_mask() { return reg_index<L>(kNR - 1); }

template <int L>
__device__ __forceinline__ uint32_t fixed_index(int lane, int warp)
{
    uint32_t t = 0;
#pragma unroll
    for (int b = 0; b < 5; b++) t |= uint32_t((lane >> b) & 1) << lane_coord(L, b);
#pragma unroll
    for (int w = 0; w < kSW; w++) t |= uint32_t((warp >> w) & 1) << warp_coord(L, w);
    return t;
}

// Slab slot of tile index t (8-byte slots; a bank pair is slot bits 0..3): bits
// 0, 1, 2, 3 XOR bits 6, 7, 8, 5. In each layout the lanes of a warp access (its
// register index fixed) differ in 5 coordinates whose images span bits 0..3, so
// each access is the minimum two wavefronts. The map is linear over GF(2):
// slot(a | b) = slot(a) ^ slot(b) for disjoint a, b.
__host__ __device__ constexpr uint32_t span_slot(uint32_t t)
{
    return t ^ ((t >> 6) & 1u) ^ (((t >> 7) & 1u) << 1) ^ (((t >> 8) & 1u) << 2) ^ (((t >> 5) & 1u) << 3);
}

// Real-address offset of tile index t.
__device__ __forceinline__ uint64_t real_of(uint32_t t, const uint8_t *pos)
{
    uint64_t o = 0;
#pragma unroll
    for (int k = 0; k < kT; k++)
        if ((t >> k) & 1) o |= 1ULL << pos[k];
    return o;
}

template <int LA, int LB>
__device__ __forceinline__ void exchange(float2 (&x)[kNR], float2 *slab, int lane, int warp)
{
    const uint32_t sa = span_slot(fixed_index<LA>(lane, warp)), sb = span_slot(fixed_index<LB>(lane, warp));
    __syncthreads();  // the slab's previous reads are done
#pragma unroll
    for (int j = 0; j < kNR; j++) slab[sa ^ span_slot(reg_index<LA>(j))] = x[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kNR; j++) x[j] = slab[sb ^ span_slot(reg_index<LB>(j))];
}

// The rotations of layout L's register coordinates that are in `mask`, each with
// one coefficient factored out (SpanDev): one paired FMA per amplitude.
template <int L>
__device__ __forceinline__ void rotate(float2 (&x)[kNR], const float2 *rot, uint32_t mask)
{
#pragma unroll
    for (int r = 0; r < kR; r++) {
        const int k = reg_coord(L, r);
        if (!((mask >> k) & 1)) continue;
        const float2 cm = rot[k];
        const float2 q = make_float2(cm.x, cm.x);
        if (cm.y == 0.0f) {  // x' = x - tau y, y' = y + tau x
            const float2 nq = make_float2(-cm.x, -cm.x);
#pragma unroll
            for (int j = 0; j < kNR; j++) {
                if ((j >> r) & 1) continue;
                const float2 lo = x[j], hi = x[j | (1 << r)];
                x[j] = __ffma2_rn(nq, hi, lo);
                x[j | (1 << r)] = __ffma2_rn(q, lo, hi);
            }
        } else {  // x' = mu x - y, y' = x + mu y
#pragma unroll
            for (int j = 0; j < kNR; j++) {
                if ((j >> r) & 1) continue;
                const float2 lo = x[j], hi = x[j | (1 << r)];
                x[j] = __ffma2_rn(q, lo, make_float2(-hi.x, -hi.y));
                x[j | (1 << r)] = __ffma2_rn(q, hi, lo);
            }
        }
    }
}

// A window's phase at a thread's amplitudes in layout L for one tile, in a form
// that needs few registers while the amplitudes are live: linear windows give
// one factor per thread (times rowf[j] per register pattern); others give the
// thread's constant and its 5 register coefficients in 32-bit turns (register x
// register terms come from qreg[j]). setup runs before the tile's loads.
struct SpanWin {
    float2 f;
    uint32_t a32, w32[kR];
};

template <int L, bool LINEAR>
__device__ __forceinline__ SpanWin span_window_setup(const uint8_t *blob, const DiagDev &dd, const float2 *s_exp,
                                                     uint64_t base, int lane, int warp)
{
    constexpr uint32_t RM = reg_mask<L>();
    const uint32_t fix = fixed_index<L>(lane, warp);
    const QuadTerm *cr = reinterpret_cast<const QuadTerm *>(blob + dd.off_cross);
    const LinTerm *ol = reinterpret_cast<const LinTerm *>(blob + dd.off_out_lin);
    const QuadTerm *oq = reinterpret_cast<const QuadTerm *>(blob + dd.off_out_quad);
    const uint32_t *kidx = reinterpret_cast<const uint32_t *>(blob + dd.off_kidx);
    // coefficient of each tile coordinate given the tile's out-of-tile bits (lane k)
    int64_t da = 0, K = 0;
    if (lane < kT) {
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
    for (int k = 0; k < kT; k++) {
        const int64_t dk = __shfl_sync(0xffffffffu, da, k);
        if (!((RM >> k) & 1) && ((fix >> k) & 1)) acc += dk;
    }
    SpanWin sw;
    if constexpr (LINEAR) {
        sw.f = phase_factor(s_exp, acc);
        return sw;
    }
    int64_t w[kR];
#pragma unroll
    for (int r = 0; r < kR; r++) w[r] = __shfl_sync(0xffffffffu, da, reg_coord(L, r));
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
        for (int r = 0; r < kR; r++)
            if (uint32_t(reg_coord(L, r)) == reg) w[r] += t.coef;
    }
    sw.a32 = turns32(acc);
#pragma unroll
    for (int r = 0; r < kR; r++) sw.w32[r] = turns32(w[r]);
    return sw;
}

template <bool LINEAR>
__device__ __forceinline__ void span_window_apply(float2 (&x)[kNR], const SpanWin &sw, const float2 *rowf,
                                                  const int64_t *qreg, const float2 *s_exp)
{
    if constexpr (LINEAR) {
#pragma unroll
        for (int j = 0; j < kNR; j++) x[j] = cmul(x[j], cmul(sw.f, rowf[j]));
    } else {
        uint32_t a32 = sw.a32;
#pragma unroll
        for (int jj = 0; jj < kNR; jj++) {
            const int gj = jj ^ (jj >> 1);
            if (jj > 0) {
                const int fb = ctz_const(jj);
                a32 += ((gj >> fb) & 1) ? sw.w32[fb] : 0u - sw.w32[fb];
            }
            x[gj] = cmul(x[gj], phase_factor32(s_exp, a32 + turns32(qreg[gj])));
        }
    }
}

// WIN: 0 no window, 1 windows with linear terms only, 2 any windows (quadratic
// terms; no multi-bit selectors). Two CTAs share an SM; each works on one tile at a
// time: loads in layout A, the windows' per-tile parts computed before the loads
// (few registers stay live across the tile), exchanges through the slab, stores
// from layout B.
template <bool LOW, int WIN>
__global__ void __launch_bounds__(kSpanThreads, 2) span_kernel(const uint8_t *__restrict__ blob, uint64_t soff,
                                                              uint64_t toff, float2 *__restrict__ state)
{
    extern __shared__ __align__(16) float2 s_slab[];  // 2^13 slots
    __shared__ float2 s_exp[WIN ? (1 << kExpTableBits) : 1];  // WIN != 0
    __shared__ float2 s_rot[kT];
    __shared__ uint64_t s_roff[2][kNR];  // real offsets of the register patterns: layout A (loads), B (stores)
    __shared__ uint8_t s_pos[16];
    __shared__ int64_t s_qreg[2][kNR];   // window 0 in layout A, window 1 in layout B
    __shared__ float2 s_rowf[2][kNR];

    const SpanDev &p = *reinterpret_cast<const SpanDev *>(blob + soff);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < 16) s_pos[tid] = p.pos[tid];
    if (tid < kT) s_rot[tid] = make_float2(p.rot[tid][0], p.rot[tid][1]);
    if constexpr (WIN != 0) {
        const float2 *tab = reinterpret_cast<const float2 *>(blob + toff);
        for (int i = tid; i < (1 << kExpTableBits); i += kSpanThreads) s_exp[i] = tab[i];
    }
    __syncthreads();
    if (tid < 2 * kNR) {
        const int L = tid >> 5, j = tid & 31;
        s_roff[L][j] = real_of(L ? reg_index<2>(j) : reg_index<0>(j), s_pos);
    }
    if (WIN && tid >= 2 * kNR && tid < 4 * kNR) {
        // tile-independent window parts: the register x register quadratic terms and,
        // for linear windows, the per-pattern factors
        const int d = (tid - 2 * kNR) >> 5, j = tid & 31;
        const uint64_t ow = d ? p.off_post : p.off_pre;
        int64_t qa = 0, lb = 0;
        if (ow) {
            const DiagDev &dd = *reinterpret_cast<const DiagDev *>(blob + ow);
            const uint32_t t = d ? reg_index<2>(j) : reg_index<0>(j);
            const QuadTerm *iq = reinterpret_cast<const QuadTerm *>(blob + dd.off_in_quad);
            for (uint32_t q = 0; q < dd.n_in_quad; q++)
                if (((t >> iq[q].i) & 1) && ((t >> iq[q].j) & 1)) qa += iq[q].coef;
            for (int k = 0; k < kT; k++)
                if ((t >> k) & 1) lb += dd.lin_in[k];
        }
        s_qreg[d][j] = qa;
        s_rowf[d][j] = phase_factor(s_exp, lb);
    }
    __syncthreads();

    const uint64_t offA = real_of(fixed_index<0>(lane, warp), s_pos);
    const uint64_t offB = real_of(fixed_index<2>(lane, warp), s_pos);
    const uint32_t gm = p.gates;
    const uint32_t gA = gm & reg_mask<0>();
    const uint32_t gAp = LOW ? (gm & reg_mask<1>() & ~gA) : 0u;
    const uint32_t gB = gm & reg_mask<2>() & ~gA & ~gAp;
    // the rotations' common factor: into a linear window's per-thread factor where
    // there is one, else one multiply before the store
    const float scale = p.scale;
    const bool scale_pre = WIN == 1 && p.off_pre != 0;
    const bool scale_post = WIN == 1 && !scale_pre && p.off_post != 0;
    const bool scale_end = !scale_pre && !scale_post;
    const uint64_t ntiles = p.ntiles;

    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        uint64_t base;
        if constexpr (LOW) {
            base = tile << kT;
        } else {
            base = tile;  // zeros inserted at the tile's real bits (ascending)
#pragma unroll
            for (int k = 0; k < kT; k++) {
                const uint32_t b = s_pos[k];
                base = ((base >> b) << (b + 1)) | (base & ((1ULL << b) - 1ULL));
            }
        }
        [[maybe_unused]] SpanWin wpre, wpost;
        if constexpr (WIN != 0) {
            if (p.off_pre) {
                wpre = span_window_setup<0, WIN == 1>(blob, *reinterpret_cast<const DiagDev *>(blob + p.off_pre), s_exp,
                                                      base, lane, warp);
                if (scale_pre) wpre.f = make_float2(wpre.f.x * scale, wpre.f.y * scale);
            }
            if (p.off_post) {
                wpost = span_window_setup<2, WIN == 1>(blob, *reinterpret_cast<const DiagDev *>(blob + p.off_post),
                                                       s_exp, base, lane, warp);
                if (scale_post) wpost.f = make_float2(wpost.f.x * scale, wpost.f.y * scale);
            }
        }
        float2 x[kNR];
        const float2 *src = state + base + offA;
#pragma unroll
        for (int j = 0; j < kNR; j++) x[j] = __ldcs(src + s_roff[0][j]);
        if constexpr (WIN != 0) {
            if (p.off_pre) span_window_apply<WIN == 1>(x, wpre, s_rowf[0], s_qreg[0], s_exp);
        }
        rotate<0>(x, s_rot, gA);
        if constexpr (LOW) {
            exchange<0, 1>(x, s_slab, lane, warp);
            rotate<1>(x, s_rot, gAp);
            exchange<1, 2>(x, s_slab, lane, warp);
        } else {
            exchange<0, 2>(x, s_slab, lane, warp);
        }
        rotate<2>(x, s_rot, gB);
        if constexpr (WIN != 0) {
            if (p.off_post) span_window_apply<WIN == 1>(x, wpost, s_rowf[1], s_qreg[1], s_exp);
        }
        if (scale_end) {
            const float2 sc = make_float2(scale, scale);
#pragma unroll
            for (int j = 0; j < kNR; j++) x[j] = __fmul2_rn(sc, x[j]);
        }
        float2 *dst = state + base + offB;
#pragma unroll
        for (int j = 0; j < kNR; j++) __stcs(dst + s_roff[1][j], x[j]);
    }
}

template <bool LOW, int WIN>
cudaError_t launch_span(const uint8_t *dblob, uint64_t soff, uint64_t toff, uint64_t ntiles, float2 *state, int sms,
                        cudaStream_t st)
{
    auto kern = span_kernel<LOW, WIN>;
    const size_t smem = kTileBytes;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSpanThreads, smem);
    if (per_sm < 1) per_sm = 1;
    const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(sms) * uint64_t(per_sm))));
    kern<<<grid, kSpanThreads, smem, st>>>(dblob, soff, toff, state);
    return cudaGetLastError();
}

}  // namespace

int span_tile_bits() { return kT; }

// Coordinates each layout holds in registers: a gate on coordinate k runs in the
// first layout of the pass whose registers include k (strided: A, B; low: A, A', B).
bool span_coverable(uint32_t gates, bool low)
{
    const uint32_t cover = reg_mask<0>() | reg_mask<2>() | (low ? reg_mask<1>() : 0u);
    return (gates & ~cover) == 0;
}

cudaError_t run_span(const uint8_t *dblob, uint64_t soff, uint64_t toff, uint64_t ntiles, bool low, int win,
                     void *state, DevStatus *, int sms, cudaStream_t st)
{
    float2 *s = static_cast<float2 *>(state);
    switch ((low ? 3 : 0) + win) {
    case 0: return launch_span<false, 0>(dblob, soff, toff, ntiles, s, sms, st);
    case 1: return launch_span<false, 1>(dblob, soff, toff, ntiles, s, sms, st);
    case 2: return launch_span<false, 2>(dblob, soff, toff, ntiles, s, sms, st);
    case 3: return launch_span<true, 0>(dblob, soff, toff, ntiles, s, sms, st);
    case 4: return launch_span<true, 1>(dblob, soff, toff, ntiles, s, sms, st);
    case 5: return launch_span<true, 2>(dblob, soff, toff, ntiles, s, sms, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace zxh
