// u3pass.cu -- the U3-batch pass (sm_100a), fast form.
//
// One pass applies up to 8 fused single-qubit gates (and, fused around them, small
// diagonal windows) to the whole state with one read and one write of every
// amplitude. The reference runs one full grid sweep per fused gate with a
// cooperative grid.sync() between them (u3_block_batch_kernel_cuda,
// src/zxh/src/kernel/kernel_cuda.cu:390-423).
//
// A tile is 2^T amplitudes: 2^c contiguous ones times 2^h strided chunks, moved
// global <-> shared by TMA bulk copies (cp.async.bulk, double-buffered, mbarrier
// completion, bounded waits). Inside the tile the amplitudes are worked on in
// registers: tile coordinates 0..4 are the lanes of a warp (gates there exchange
// partners with shfl.xor), in each shared-memory round R further coordinates are
// a thread's registers (gates there are register-local 2x2 updates) and 3 select
// the warp. Diagonal windows fused into the pass are evaluated per amplitude as a
// polynomial in 64-bit fixed-point turns (Gray-code walk over the register bits)
// and one table-plus-Taylor exp.
#include "core.h"
#include "dev.cuh"
#include "host.h"
#include "sampler.h"

#include <algorithm>
#include <cuda_runtime.h>

namespace zxh {

namespace {

template <typename E>
struct FastCfg;
template <>
struct FastCfg<float2> {
    static constexpr int R = 4;  // register coordinates per round: T = 5 + 3 + 4 = 12
};
template <>
struct FastCfg<double2> {
    static constexpr int R = 3;  // T = 11
};

__device__ __forceinline__ uint64_t pdep_bits(uint64_t x, uint64_t mask)
{
    uint64_t r = 0;
    for (uint64_t bb = 1; mask; bb += bb) {
        const uint64_t low = mask & (0 - mask);
        if (x & bb) r |= low;
        mask &= mask - 1;
    }
    return r;
}

__device__ __forceinline__ uint64_t fchunk_base(const TileDev &g, uint64_t r, uint32_t j)
{
    uint64_t a = r;
    for (uint32_t b = 0; b < g.h; b++)
        if ((j >> b) & 1) a |= 1ULL << g.pos[g.c + b];
    return a;
}

// Bulk copies of one tile, spread over all threads: thread t moves chunks t,
// t + 256, ...; each warp announces its own byte count on the stage's mbarrier
// (initialised with one arrival per warp), so no cross-warp ordering is needed.
template <typename E>
__device__ __forceinline__ void fload(const TileDev &g, const E *state, E *buf, uint64_t r, uint64_t *bar, int tid)
{
    const uint32_t nchunk = 1u << g.h;
    const uint32_t cbytes = uint32_t(sizeof(E)) << g.c;
    const int warp = tid >> 5, lane = tid & 31;
    uint32_t mine = 0;  // chunks of this warp
    for (uint32_t j0 = uint32_t(warp) * 32; j0 < nchunk; j0 += kThreads) mine += min(32u, nchunk - j0);
    if (lane == 0) mbar_arrive_expect_tx(bar, mine * cbytes);
    __syncwarp();
    for (uint32_t j = uint32_t(tid); j < nchunk; j += kThreads)
        bulk_g2s(buf + (size_t(j) << g.c), state + fchunk_base(g, r, j), cbytes, bar);
}

template <typename E>
__device__ __forceinline__ void fstore(const TileDev &g, E *state, const E *buf, uint64_t r, int tid)
{
    const uint32_t nchunk = 1u << g.h;
    const uint32_t cbytes = uint32_t(sizeof(E)) << g.c;
    for (uint32_t j = uint32_t(tid); j < nchunk; j += kThreads)
        bulk_s2g(state + fchunk_base(g, r, j), buf + (size_t(j) << g.c), cbytes);
    bulk_commit();
}

// Per-tile coefficients of a fused window, computed by one warp: lane k < T sums
// the cross terms of tile coordinate k, all lanes share the out-of-tile constant.
__device__ __forceinline__ void window_tile_params(const uint8_t *blob, const DiagDev &d, uint64_t r, uint32_t T,
                                                   int lane, int64_t *da, int64_t *K)
{
    const QuadTerm *cr = reinterpret_cast<const QuadTerm *>(blob + d.off_cross);
    const LinTerm *ol = reinterpret_cast<const LinTerm *>(blob + d.off_out_lin);
    const QuadTerm *oq = reinterpret_cast<const QuadTerm *>(blob + d.off_out_quad);
    const uint32_t *kidx = reinterpret_cast<const uint32_t *>(blob + d.off_kidx);
    int64_t a = 0;
    if (lane < int(T)) {
        a = d.lin_in[lane];
        for (uint32_t q = kidx[lane]; q < kidx[lane + 1]; q++) {
            const QuadTerm t = cr[q];
            if ((r >> t.j) & 1) a += t.coef;
        }
        da[lane] = a;
    }
    int64_t kp = 0;
    for (uint32_t q = uint32_t(lane); q < d.n_out_lin; q += 32)
        if ((r >> ol[q].bit) & 1) kp += ol[q].coef;
    for (uint32_t q = uint32_t(lane); q < d.n_out_quad; q += 32) {
        const QuadTerm t = oq[q];
        if (((r >> t.i) & 1) && ((r >> t.j) & 1)) kp += t.coef;
    }
    kp = warp_sum_i64(kp);
    if (lane == 0) *K = kp + d.c0;
}

}  // namespace

namespace {

template <typename E, int R>
__device__ __forceinline__ void apply_window(E (&x)[1 << R], const E *s_exp, int64_t A, const int64_t (&w)[R],
                                             const int64_t *qreg)
{
    int64_t acc = A;
#pragma unroll
    for (int jj = 0; jj < (1 << R); jj++) {
        const int gj = jj ^ (jj >> 1);
        if (jj > 0) {
            const int fb = __ffs(jj) - 1;  // a run-time index: w stays in local memory, off the registers
            acc += ((gj >> fb) & 1) ? w[fb] : -w[fb];
        }
        x[gj] = cmul(x[gj], phase_factor(s_exp, acc + qreg[gj]));
    }
}

template <typename E>
__device__ __forceinline__ E shfl_xor_e(E v, int m);
template <>
__device__ __forceinline__ float2 shfl_xor_e(float2 v, int m)
{
    return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
template <>
__device__ __forceinline__ double2 shfl_xor_e(double2 v, int m)
{
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// a*x + b*y for complex a, b given as (re, im) pairs
template <typename E, typename RT>
__device__ __forceinline__ E cmad2(RT ar, RT ai, E x, RT br, RT bi, E y)
{
    E o;
    o.x = ar * x.x - ai * x.y + br * y.x - bi * y.y;
    o.y = ar * x.y + ai * x.x + br * y.y + bi * y.x;
    return o;
}

// 2x2 gate on register bit RR of every row pair: compile-time positions keep the
// amplitudes in registers. REAL: the matrix has no imaginary parts (a rotation
// split off a U3 by the planner), half the multiply-adds.
template <int RR, int NR, int V, bool REAL, typename VT, typename RT>
__device__ __forceinline__ void reg_gate(VT (&x)[NR], const RT *u)
{
    using E = decltype(vget(x[0], 0));
    const RT m00r = u[0], m00i = u[1], m01r = u[2], m01i = u[3];
    const RT m10r = u[4], m10i = u[5], m11r = u[6], m11i = u[7];
#pragma unroll
    for (int j = 0; j < NR; j++) {
        if ((j >> RR) & 1) continue;
#pragma unroll
        for (int v = 0; v < V; v++) {
            const E lo = vget(x[j], v), hi = vget(x[j | (1 << RR)], v);
            if constexpr (REAL) {
                vset(x[j], v, rmad2(m00r, lo, m01r, hi));
                vset(x[j | (1 << RR)], v, rmad2(m10r, lo, m11r, hi));
            } else {
                vset(x[j], v, cmad2(m00r, m00i, lo, m01r, m01i, hi));
                vset(x[j | (1 << RR)], v, cmad2(m10r, m10i, lo, m11r, m11i, hi));
            }
        }
    }
}

// One gate on tile coordinate c of a row-pass thread's amplitudes: c < LV is the
// vector bit, c < F a lane bit (partner by shfl.xor), otherwise register bit c - F.
template <int R, int V, int LV, int F, bool REAL = false, typename VT, typename RT>
__device__ __forceinline__ void row_gate(VT (&x)[1 << R], uint32_t c, const RT *u, int lane)
{
    using E = decltype(vget(x[0], 0));
    constexpr int NR = 1 << R;
    if (int(c) < LV) {
        const RT m00r = u[0], m00i = u[1], m01r = u[2], m01i = u[3];
        const RT m10r = u[4], m10i = u[5], m11r = u[6], m11i = u[7];
#pragma unroll
        for (int j = 0; j < NR; j++) {
            const E lo = vget(x[j], 0), hi = vget(x[j], V - 1);
            if constexpr (REAL) {
                vset(x[j], 0, rmad2(m00r, lo, m01r, hi));
                vset(x[j], V - 1, rmad2(m10r, lo, m11r, hi));
            } else {
                vset(x[j], 0, cmad2(m00r, m00i, lo, m01r, m01i, hi));
                vset(x[j], V - 1, cmad2(m10r, m10i, lo, m11r, m11i, hi));
            }
        }
    } else if (int(c) < F) {
        const int lb = int(c) - LV;
        const bool hb = (lane >> lb) & 1;
        const RT ar = hb ? u[6] : u[0], ai = hb ? u[7] : u[1];
        const RT br = hb ? u[4] : u[2], bi = hb ? u[5] : u[3];
#pragma unroll
        for (int j = 0; j < NR; j++)
#pragma unroll
            for (int v = 0; v < V; v++) {
                const E mine = vget(x[j], v);
                const E pt = shfl_xor_e(mine, 1 << lb);
                if constexpr (REAL) vset(x[j], v, rmad2(ar, mine, br, pt));
                else vset(x[j], v, cmad2(ar, ai, mine, br, bi, pt));
            }
    } else {
        switch (int(c) - F) {
        case 0: reg_gate<0, NR, V, REAL>(x, u); break;
        case 1: if constexpr (R > 1) reg_gate<(R > 1 ? 1 : 0), NR, V, REAL>(x, u); break;
        case 2: if constexpr (R > 2) reg_gate<(R > 2 ? 2 : 0), NR, V, REAL>(x, u); break;
        case 3: if constexpr (R > 3) reg_gate<(R > 3 ? 3 : 0), NR, V, REAL>(x, u); break;
        case 4: if constexpr (R > 4) reg_gate<(R > 4 ? 4 : 0), NR, V, REAL>(x, u); break;
        default: break;
        }
    }
}

template <typename E>
__global__ void __launch_bounds__(kThreads, 2) fast_tile_kernel(const uint8_t *__restrict__ blob, uint64_t foff,
                                                             uint64_t toff, E *__restrict__ state, DevStatus *status)
{
    using RT = typename ET<E>::R;
    constexpr int R = FastCfg<E>::R;
    constexpr int NR = 1 << R;
    const FastDev &f = *reinterpret_cast<const FastDev *>(blob + foff);
    const TileDev g = f.g;
    const uint32_t T = g.T;
    const uint32_t tile_elems = 1u << T;
    extern __shared__ __align__(128) unsigned char dsm[];
    E *bufs[2] = {reinterpret_cast<E *>(dsm), reinterpret_cast<E *>(dsm) + tile_elems};
    E *s_exp = reinterpret_cast<E *>(dsm) + 2 * tile_elems;
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint64_t s_r[2];
    __shared__ int64_t s_da[2][kMaxTileBits];
    __shared__ int64_t s_K[2];
    __shared__ int64_t s_qreg[2][NR];
    __shared__ RT s_u[kFastMaxGates][8];
    __shared__ uint32_t s_gc[kFastMaxGates];

    const int tid = int(threadIdx.x), lane = tid & 31, warp = tid >> 5;
    const uint32_t ngates = f.ngates, nrounds = f.nrounds;
    const uint64_t offw0 = f.off_pre, offw1 = f.off_post;
    const FastGateDev *gates = reinterpret_cast<const FastGateDev *>(blob + f.off_gates);

    if (offw0 || offw1) {
        const E *tab = reinterpret_cast<const E *>(blob + toff);
        for (int i = tid; i < (1 << kExpTableBits); i += kThreads) s_exp[i] = tab[i];
    }
    if (tid < int(ngates)) s_gc[tid] = gates[tid].coord | (gates[tid].round << 8);

    // register x register quadratic part of each window, for the round it runs in
#pragma unroll
    for (int d = 0; d < 2; d++) {
        const uint64_t ow = d ? offw1 : offw0;
        if (!ow || tid >= NR) continue;
        const DiagDev &dd = *reinterpret_cast<const DiagDev *>(blob + ow);
        const QuadTerm *iq = reinterpret_cast<const QuadTerm *>(blob + dd.off_in_quad);
        const RoundDev rd = f.rounds[d == 0 ? 0 : nrounds - 1];
        int64_t acc = 0;
        for (uint32_t q = 0; q < dd.n_in_quad; q++) {
            const QuadTerm t = iq[q];
            int a = -1, b = -1;
            for (int r = 0; r < R; r++) {
                if (t.i == rd.rc[r]) a = r;
                if (t.j == rd.rc[r]) b = r;
            }
            if (a >= 0 && b >= 0 && ((tid >> a) & 1) && ((tid >> b) & 1)) acc += t.coef;
        }
        s_qreg[d][tid] = acc;
    }

    if (tid == 0) {
        mbar_init(&mbar[0], kThreads / 32);
        mbar_init(&mbar[1], kThreads / 32);
        s_r[0] = pdep_bits(blockIdx.x, g.free_mask);
        fence_mbar_init();
    }
    __syncthreads();

    uint64_t tidx = blockIdx.x;
    if (tidx >= g.ntiles) return;
    fload(g, state, bufs[0], s_r[0], &mbar[0], tid);

    for (uint32_t k = 0;; k++, tidx += gridDim.x) {
        if (tidx >= g.ntiles) break;
        const int s = int(k & 1);
        const uint64_t nxt = tidx + gridDim.x;
        // the block gives up as one (no thread left behind at a barrier); only this
        // tile's copy can be in flight then, and each thread waits for it (bounded)
        if (__syncthreads_or(!mbar_wait_bounded(&mbar[s], (k >> 1) & 1))) {
            if (tid == 0) report(status, kErrTimeout, 3, tidx);
            (void)mbar_wait_bounded(&mbar[s], (k >> 1) & 1);
            bulk_wait0();
            return;
        }
        bulk_wait_read0();  // this thread's stores of the previous tile (other stage) have read it
        if (tid == 0 && nxt < g.ntiles) s_r[s ^ 1] = pdep_bits(nxt, g.free_mask);
        E *buf = bufs[s];
        const uint64_t r = s_r[s];

        // per-tile parameters: warp 0 / 1 the fused windows, warp 2 the gate selectors
        if (warp == 0 && offw0)
            window_tile_params(blob, *reinterpret_cast<const DiagDev *>(blob + offw0), r, T, lane, s_da[0], &s_K[0]);
        if (warp == 1 && offw1)
            window_tile_params(blob, *reinterpret_cast<const DiagDev *>(blob + offw1), r, T, lane, s_da[1], &s_K[1]);
        if (warp == 2 && lane < int(ngates)) {
            const FastGateDev &gg = gates[lane];
            const int beta = int(gg.beta) ^ par64(gg.alpha_out & r);
            // with beta = 1 the odd partner sits at bit value 0: swap the roles
            const int p[8] = {0, 1, 2, 3, 4, 5, 6, 7};
            const int q[8] = {6, 7, 4, 5, 2, 3, 0, 1};
#pragma unroll
            for (int i = 0; i < 8; i++) s_u[lane][i] = RT(gg.u[beta ? q[i] : p[i]]);
        }
        __syncthreads();
        if (nxt < g.ntiles) fload(g, state, bufs[s ^ 1], s_r[s ^ 1], &mbar[s ^ 1], tid);

        for (uint32_t rnd = 0; rnd < nrounds; rnd++) {
            const RoundDev rd = f.rounds[rnd];
            const uint32_t ebase = uint32_t(lane) | (uint32_t(warp & 1) << rd.oc[0]) |
                                   (uint32_t((warp >> 1) & 1) << rd.oc[1]) | (uint32_t((warp >> 2) & 1) << rd.oc[2]);
            uint32_t off[NR];
#pragma unroll
            for (int j = 0; j < NR; j++) {
                uint32_t o = 0;
#pragma unroll
                for (int rr = 0; rr < R; rr++)
                    if ((j >> rr) & 1) o |= 1u << rd.rc[rr];
                off[j] = ebase | o;
            }
            E x[NR];
#pragma unroll
            for (int j = 0; j < NR; j++) x[j] = buf[off[j]];

            // fused window d for this thread's amplitudes (fixed bits: lane and warp
            // coordinates; register bits: rd.rc)
            auto window = [&](int d, uint64_t ow) {
                const DiagDev &dd = *reinterpret_cast<const DiagDev *>(blob + ow);
                const QuadTerm *iq = reinterpret_cast<const QuadTerm *>(blob + dd.off_in_quad);
                int64_t A = s_K[d];
                int64_t w[R];
#pragma unroll
                for (int kk = 0; kk < 5; kk++)
                    if ((lane >> kk) & 1) A += s_da[d][kk];
#pragma unroll
                for (int i = 0; i < 3; i++)
                    if ((warp >> i) & 1) A += s_da[d][rd.oc[i]];
#pragma unroll
                for (int rr = 0; rr < R; rr++) w[rr] = s_da[d][rd.rc[rr]];
                // quadratic terms with a fixed bit set: fixed x fixed -> A, fixed x register -> w
                for (uint32_t q = 0; q < dd.n_in_quad; q++) {
                    const QuadTerm t = iq[q];
                    int bi = -1, bj = -1, ri = -1, rj = -1;  // bit value of a fixed coordinate, or register slot
                    if (t.i < 5) bi = (lane >> t.i) & 1;
                    if (t.j < 5) bj = (lane >> t.j) & 1;
#pragma unroll
                    for (int i = 0; i < 3; i++) {
                        if (t.i == rd.oc[i]) bi = (warp >> i) & 1;
                        if (t.j == rd.oc[i]) bj = (warp >> i) & 1;
                    }
#pragma unroll
                    for (int rr = 0; rr < R; rr++) {
                        if (t.i == rd.rc[rr]) ri = rr;
                        if (t.j == rd.rc[rr]) rj = rr;
                    }
                    if (bi == 1 && bj == 1) A += t.coef;
                    else if (bi == 1 && rj >= 0) {
#pragma unroll
                        for (int rr = 0; rr < R; rr++)
                            if (rr == rj) w[rr] += t.coef;
                    } else if (bj == 1 && ri >= 0) {
#pragma unroll
                        for (int rr = 0; rr < R; rr++)
                            if (rr == ri) w[rr] += t.coef;
                    }
                }
                apply_window<E, R>(x, s_exp, A, w, s_qreg[d]);
            };
            if (offw0 && rnd == 0) window(0, offw0);

            for (uint32_t gi = 0; gi < ngates; gi++) {
                const uint32_t gc = s_gc[gi];
                if ((gc >> 8) != rnd) continue;
                const uint32_t c = gc & 255u;
                // lane coordinates 0..4 stay; a register coordinate maps to its slot
                uint32_t cc = c;
                if (c >= 5) {
                    cc = 5 + R;  // not in this round (cannot happen for a planned gate)
#pragma unroll
                    for (int rr = 0; rr < R; rr++)
                        if (rd.rc[rr] == c) cc = 5 + uint32_t(rr);
                }
                row_gate<R, 1, 0, 5>(x, cc, &s_u[gi][0], lane);
            }

            if (offw1 && rnd == nrounds - 1) window(1, offw1);
#pragma unroll
            for (int j = 0; j < NR; j++) buf[off[j]] = x[j];
            __syncthreads();
        }

        fence_proxy_async();
        __syncthreads();
        fstore(g, state, buf, r, tid);
    }
    bulk_wait0();
}

}  // namespace

int fast_tile_bits(int elem_bytes) { return 8 + (elem_bytes == 8 ? FastCfg<float2>::R : FastCfg<double2>::R); }

int fast_reg_bits(int elem_bytes) { return elem_bytes == 8 ? FastCfg<float2>::R : FastCfg<double2>::R; }

cudaError_t run_fast_tile(const uint8_t *dblob, uint64_t foff, uint64_t toff, uint64_t ntiles, int elem_bytes,
                          void *state, DevStatus *status, int sms, cudaStream_t st)
{
    const int T = fast_tile_bits(elem_bytes);
    const size_t smem = 2 * (size_t(elem_bytes) << T) + size_t(elem_bytes) * (1u << kExpTableBits);
    int per_sm = 1;
    cudaError_t e;
    if (elem_bytes == 8) {
        e = cudaFuncSetAttribute(fast_tile_kernel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fast_tile_kernel<float2>, kThreads, smem);
    } else {
        e = cudaFuncSetAttribute(fast_tile_kernel<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fast_tile_kernel<double2>, kThreads, smem);
    }
    if (per_sm < 1) per_sm = 1;
    const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(sms) * uint64_t(per_sm))));
    if (elem_bytes == 8)
        fast_tile_kernel<float2><<<grid, kThreads, smem, st>>>(dblob, foff, toff, static_cast<float2 *>(state), status);
    else
        fast_tile_kernel<double2><<<grid, kThreads, smem, st>>>(dblob, foff, toff, static_cast<double2 *>(state), status);
    return cudaGetLastError();
}

}  // namespace zxh

// ---------------------------------------------------------------------------
// Strided high-qubit pass: no shared-memory staging; a thread's registers span R
// arbitrary (high) bits, so one pass applies up to R gates on any bits with each
// amplitude read and written once.

namespace zxh {

namespace {

// Row-pass shapes: VT is what one lane loads per row (V amplitudes), R the register
// bits. Variant 0 / 1 of each type are picked by the planner's row_wide knob.
template <typename E, int W>
struct RowCfg;
template <>
struct RowCfg<float2, 0> {
    using VT = float4;
    static constexpr int V = 2, R = 4;  // 16 rows of 512 bytes per warp
};
template <>
struct RowCfg<float2, 1> {
    using VT = float2;
    static constexpr int V = 1, R = 5;  // 32 rows of 256 bytes per warp
};
template <>
struct RowCfg<double2, 0> {
    using VT = double2;
    static constexpr int V = 1, R = 3;  // 8 rows of 512 bytes per warp
};
template <>
struct RowCfg<double2, 1> {
    using VT = double2;
    static constexpr int V = 1, R = 4;
};


// A window with linear terms only: the phase is K(item) + A(lane, vector slot) +
// B(row), so each amplitude takes one product of two factors: e^{i (K + A)} per
// thread and item, e^{i B} per row from rowf (per CTA, shared). apply(row, v,
// factor) is called for every amplitude.
template <int F, int LV, int R, int V, typename E, typename Apply>
__device__ __forceinline__ void row_window_linear(const uint8_t *blob, const DiagDev &dd, const E *rowf,
                                                  const E *s_exp, uint64_t base, int lane, Apply &&apply)
{
    constexpr int NR = 1 << R;
    const LinTerm *ol = reinterpret_cast<const LinTerm *>(blob + dd.off_out_lin);
    int64_t K = 0;
    for (uint32_t q = uint32_t(lane); q < dd.n_out_lin; q += 32)
        if ((base >> ol[q].bit) & 1) K += ol[q].coef;
    K = warp_sum_i64(K) + dd.c0;
    E fa[V];
#pragma unroll
    for (int v = 0; v < V; v++) {
        const uint32_t e = uint32_t(v) | (uint32_t(lane) << LV);
        int64_t a = K;
#pragma unroll
        for (int k = 0; k < F; k++)
            if ((e >> k) & 1) a += dd.lin_in[k];
        fa[v] = phase_factor(s_exp, a);
    }
#pragma unroll
    for (int j = 0; j < NR; j++) {
        const E fb = rowf[j];
#pragma unroll
        for (int v = 0; v < V; v++) apply(j, v, cmul(fa[v], fb));
    }
}

// Phases of a window fused into a strided pass, at one thread's amplitudes. Tile
// coordinates are [0, F) = vector and lane bits, then F + r = register bit r;
// base holds the item's out-of-tile bits. apply(row, v, factor) is called for
// every row (in Gray-code order) and vector slot v with the phase factor.
template <int F, int LV, int R, int V, typename E, typename Apply>
__device__ __forceinline__ void row_window(const uint8_t *blob, const DiagDev &dd, const int64_t *qreg,
                                           const E *s_exp, uint64_t base, int lane, Apply &&apply)
{
    constexpr int T = F + R;
    constexpr int NR = 1 << R;
    int64_t da = 0, K = 0;
    const QuadTerm *cr = reinterpret_cast<const QuadTerm *>(blob + dd.off_cross);
    const LinTerm *ol = reinterpret_cast<const LinTerm *>(blob + dd.off_out_lin);
    const QuadTerm *oq = reinterpret_cast<const QuadTerm *>(blob + dd.off_out_quad);
    const uint32_t *kidx = reinterpret_cast<const uint32_t *>(blob + dd.off_kidx);
    if (lane < T) {
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
    K = warp_sum_i64(K) + dd.c0;
    int64_t acc[V], w[R][V];
#pragma unroll
    for (int v = 0; v < V; v++) {
        acc[v] = K;
#pragma unroll
        for (int r = 0; r < R; r++) w[r][v] = 0;
    }
    // in-tile quadratic terms touching this thread's fixed (vector / lane) bits
    const QuadTerm *iq = reinterpret_cast<const QuadTerm *>(blob + dd.off_in_quad);
    for (uint32_t q = 0; q < dd.n_in_quad; q++) {
        const QuadTerm t = iq[q];  // t.i < t.j
        if (int(t.i) >= F) continue;
#pragma unroll
        for (int v = 0; v < V; v++) {
            const uint32_t e = uint32_t(v) | (uint32_t(lane) << LV);
            if (!((e >> t.i) & 1)) continue;
            if (int(t.j) < F) {
                if ((e >> t.j) & 1) acc[v] += t.coef;
            } else {
#pragma unroll
                for (int r = 0; r < R; r++)
                    if (int(t.j) - F == r) w[r][v] += t.coef;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < F; k++) {
        const int64_t dk = __shfl_sync(0xffffffffu, da, k);
#pragma unroll
        for (int v = 0; v < V; v++)
            if (((uint32_t(v) | (uint32_t(lane) << LV)) >> k) & 1) acc[v] += dk;
    }
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int64_t dk = __shfl_sync(0xffffffffu, da, F + r);
#pragma unroll
        for (int v = 0; v < V; v++) w[r][v] += dk;
    }
    if constexpr (sizeof(E) == 8) {
        // complex64: the walk in 32-bit turns (2 pi / 2^32 resolution) and the
        // table-plus-Taylor factor without an integer-to-float conversion
        uint32_t a32[V], w32[R][V];
#pragma unroll
        for (int v = 0; v < V; v++) {
            a32[v] = turns32(acc[v]);
#pragma unroll
            for (int r = 0; r < R; r++) w32[r][v] = turns32(w[r][v]);
        }
#pragma unroll
        for (int jj = 0; jj < NR; jj++) {
            const int gj = jj ^ (jj >> 1);
            if (jj > 0) {
                const int fb = __ffs(jj) - 1;  // a run-time index: w stays in local memory, off the registers
#pragma unroll
                for (int v = 0; v < V; v++) a32[v] += ((gj >> fb) & 1) ? w32[fb][v] : 0u - w32[fb][v];
            }
            const uint32_t qr = turns32(qreg[gj]);
#pragma unroll
            for (int v = 0; v < V; v++)
                apply(gj, v, phase_factor32(reinterpret_cast<const float2 *>(s_exp), a32[v] + qr));
        }
    } else {
#pragma unroll
        for (int jj = 0; jj < NR; jj++) {
            const int gj = jj ^ (jj >> 1);
            if (jj > 0) {
                const int fb = __ffs(jj) - 1;  // a run-time index: w stays in local memory, off the registers
#pragma unroll
                for (int v = 0; v < V; v++) acc[v] += ((gj >> fb) & 1) ? w[fb][v] : -w[fb][v];
            }
            const int64_t qr = qreg[gj];
#pragma unroll
            for (int v = 0; v < V; v++) apply(gj, v, phase_factor(s_exp, acc[v] + qr));
        }
    }
}

__device__ __forceinline__ float4 as_f4(const float4 &v) { return v; }
__device__ __forceinline__ float4 as_f4(const double2 &v)
{
    return make_float4(__int_as_float(__double2loint(v.x)), __int_as_float(__double2hiint(v.x)),
                       __int_as_float(__double2loint(v.y)), __int_as_float(__double2hiint(v.y)));
}
__device__ __forceinline__ void from_f4(float4 &v, const float4 &t) { v = t; }
__device__ __forceinline__ void from_f4(double2 &v, const float4 &t)
{
    v.x = __hiloint2double(__float_as_int(t.y), __float_as_int(t.x));
    v.y = __hiloint2double(__float_as_int(t.w), __float_as_int(t.z));
}

// Swaps lane bits 0..3 with register bits 0..3 of a strided-pass thread (16-byte
// rows, 16 of them) through the warp's 16 x 32 shared-memory slots: slot of (lane
// l, row j) = j * 32 + (l ^ (j & 7)), conflict-free both ways. Afterwards thread
// L's row j holds what lane (L & 16) | j had in row L & 15. back = true undoes it.
// With 32 rows of 8 bytes all 5 lane bits swap with the 5 register bits: slot of
// (lane l, row j) = j * 32 + (l ^ j); thread L's row j then holds lane j's row L.
template <typename VT, int NR>
__device__ __forceinline__ void lane_row_transpose(VT (&x)[NR], void *tbv, int lane, bool back)
{
    if constexpr (NR == 32) {
        static_assert(sizeof(VT) == 8, "32 rows of 8 bytes");
        VT *tb = static_cast<VT *>(tbv);
#pragma unroll
        for (int j = 0; j < 32; j++) tb[back ? lane * 32 + (j ^ lane) : j * 32 + (lane ^ j)] = x[j];
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 32; j++) x[j] = tb[back ? j * 32 + (lane ^ j) : lane * 32 + (j ^ lane)];
    } else {
        static_assert(NR == 16, "16 rows of 16 bytes or 32 rows of 8 bytes");
        float4 *tb = static_cast<float4 *>(tbv);
        const int jr = lane & 15, hi = lane & 16;
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const int slot = back ? jr * 32 + (hi | (j ^ (jr & 7))) : j * 32 + (lane ^ (j & 7));
            tb[slot] = as_f4(x[j]);
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const int slot = back ? j * 32 + (lane ^ (j & 7)) : jr * 32 + (hi | (j ^ (jr & 7)));
            from_f4(x[j], tb[slot]);
        }
    }
}

// XP (the low pass): the pass also owns the lowest bits. Gates on lane bits 0..R-1
// run as register updates after lane_row_transpose (a second transpose restores
// the layout before the store); with 16-byte rows the top lane bit keeps its
// shfl.xor gate. One pass then applies gates on the F lowest bits and on R more
// with one read and one write of every amplitude.
template <typename E, int W, bool XP, bool REAL, bool WIN>
__global__ void __launch_bounds__(kThreads, 2) row_pass_kernel(const uint8_t *__restrict__ blob, uint64_t poff,
                                                            uint64_t toff, E *__restrict__ state)
{
    using VT = typename RowCfg<E, W>::VT;
    using RT = typename ET<E>::R;
    constexpr int V = RowCfg<E, W>::V;
    constexpr int LV = (V == 2) ? 1 : 0;
    constexpr int F = 5 + LV;
    constexpr int R = RowCfg<E, W>::R;
    constexpr int NR = 1 << R;
    constexpr int WARPS = kThreads / 32;
    static_assert(!XP || (R == 4 && sizeof(VT) == 16) || (R == 5 && sizeof(VT) == 8),
                  "the low pass swaps lane bits with 16 rows of 16 bytes or 32 rows of 8 bytes");
    extern __shared__ __align__(128) float4 s_xp[];  // XP: NR x 32 row slots per warp

    const RowPassDev &p = *reinterpret_cast<const RowPassDev *>(blob + poff);
    const FastGateDev *gates = reinterpret_cast<const FastGateDev *>(blob + p.off_gates);
    const uint64_t offw0 = p.off_pre, offw1 = p.off_post;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t ngates = p.ngates;
    constexpr uint32_t Rn = R;  // the planner pads the register bits to exactly R
    const uint64_t nitems = p.nitems;
    __shared__ uint32_t s_rb[8];
    if (tid < 8) s_rb[tid] = p.rb[tid];

    __shared__ E s_exp[1 << kExpTableBits];
    __shared__ RT s_u[kFastMaxGates][2][8];
    __shared__ uint32_t s_gc[kFastMaxGates];
    __shared__ int64_t s_qreg[2][NR];
    __shared__ uint64_t s_off[NR];
    __shared__ E s_rowf[2][NR];  // linear windows: e^{i B(row)}
    __shared__ int s_linear[2];

    if (WIN && (offw0 || offw1)) {
        const E *tab = reinterpret_cast<const E *>(blob + toff);
        for (int i = tid; i < (1 << kExpTableBits); i += kThreads) s_exp[i] = tab[i];
    }
    if (tid < int(ngates)) {
        const FastGateDev &gg = gates[tid];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            s_u[tid][0][i] = RT(gg.u[i]);
            s_u[tid][1][i] = RT(gg.u[i ^ 6]);  // odd partner at bit value 0: [[u11,u10],[u01,u00]]
        }
        s_gc[tid] = gg.coord;
    }
    if (tid < NR) {
        uint64_t o = 0;
        for (uint32_t r = 0; r < Rn; r++)
            if ((tid >> r) & 1) o |= 1ULL << p.rb[r];  // read once per CTA
        s_off[tid] = o;
    }

    // tile-independent parts of the windows: tile coordinates are [0, F) = vector and
    // lane bits, then F + r = register bit r
    // row-only quadratic part of each window (reg x reg coordinates): per CTA
#pragma unroll
    for (int d = 0; d < 2; d++) {
        const uint64_t ow = d ? offw1 : offw0;
        if (!ow || tid >= NR) continue;
        const DiagDev &dd = *reinterpret_cast<const DiagDev *>(blob + ow);
        const QuadTerm *iq = reinterpret_cast<const QuadTerm *>(blob + dd.off_in_quad);
        int64_t acc = 0;
        for (uint32_t q = 0; q < dd.n_in_quad; q++) {
            const QuadTerm t = iq[q];
            if (int(t.i) >= F && ((tid >> (t.i - F)) & 1) && ((tid >> (t.j - F)) & 1)) acc += t.coef;
        }
        s_qreg[d][tid] = acc;
    }
    __syncthreads();
    if (WIN) {
#pragma unroll
        for (int d = 0; d < 2; d++) {
            const uint64_t ow = d ? offw1 : offw0;
            if (!ow) continue;
            const DiagDev &dd = *reinterpret_cast<const DiagDev *>(blob + ow);
            const bool lin = dd.n_in_quad == 0 && dd.n_cross == 0 && dd.n_out_quad == 0 && dd.n_gen == 0;
            if (tid == 0) s_linear[d] = lin ? 1 : 0;
            if (lin && tid < NR) {
                int64_t b = 0;
                for (int r = 0; r < R; r++)
                    if ((tid >> r) & 1) b += dd.lin_in[F + r];
                s_rowf[d][tid] = phase_factor(s_exp, b);
            }
        }
        __syncthreads();
    }

    const uint64_t stride = uint64_t(gridDim.x) * WARPS;
    for (uint64_t item = uint64_t(blockIdx.x) * WARPS + uint64_t(warp); item < nitems; item += stride) {
        // item bits go to every real bit outside [0, F) and the register bits
        uint64_t base = item << F;
        for (uint32_t r = 0; r < Rn; r++) {
            const uint32_t b = s_rb[r];
            base = ((base >> b) << (b + 1)) | (base & ((1ULL << b) - 1ULL));
        }
        E *rowp = state + base + (uint64_t(lane) << LV);
        VT x[NR];
#pragma unroll
        for (int j = 0; j < NR; j++)
            x[j] = __ldcs(reinterpret_cast<const VT *>(rowp + s_off[j]));

        // per-item selector orientation of every gate
        int ob = 0;
        if (lane < int(ngates)) {
            const FastGateDev &gg = gates[lane];
            ob = int(gg.beta) ^ par64(gg.alpha_out & base);
        }
        const uint32_t omask = __ballot_sync(0xffffffffu, ob);

        auto window = [&](int d, uint64_t ow) {
            const DiagDev &dd = *reinterpret_cast<const DiagDev *>(blob + ow);
            if (s_linear[d])
                row_window_linear<F, LV, R, V>(blob, dd, s_rowf[d], s_exp, base, lane, [&](int j, int v, E f) {
                    vset(x[j], v, cmul(vget(x[j], v), f));
                });
            else
                row_window<F, LV, R, V>(blob, dd, s_qreg[d], s_exp, base, lane, [&](int j, int v, E f) {
                    vset(x[j], v, cmul(vget(x[j], v), f));
                });
        };
        if constexpr (WIN) {
            if (offw0) window(0, offw0);
        }
        void *tb = reinterpret_cast<unsigned char *>(s_xp) + size_t(warp) * NR * 32 * sizeof(VT);
        if constexpr (REAL) {
            // dense table (real passes): slot i holds the gate of coordinate C0 + i
            // (identity where the pass has none), so the loop unrolls with
            // compile-time coordinates and no per-gate dispatch
            constexpr int C0 = XP ? 0 : F, NS = XP ? F + R : R;
#pragma unroll
            for (int i = 0; i < NS; i++) {
                if (XP && i >= LV && i < LV + R) continue;  // lane bits 0..R-1: after the transpose
                row_gate<R, V, LV, F, true>(x, uint32_t(C0 + i), &s_u[i][(omask >> i) & 1][0], lane);
            }
            if constexpr (XP) {
                lane_row_transpose(x, tb, lane, false);
#pragma unroll
                for (int b = 0; b < R; b++)
                    row_gate<R, V, LV, F, true>(x, uint32_t(F + b), &s_u[LV + b][(omask >> (LV + b)) & 1][0], lane);
                lane_row_transpose(x, tb, lane, true);
            }
        } else {
            // XP: phase 0 runs the gates on the vector, top lane and register bits,
            // phase 1 (after the transpose) those on lane bits 0..3 as register gates
            bool swapped = false;
#pragma unroll 1
            for (int ph = 0; ph < (XP ? 2 : 1); ph++) {
                if constexpr (XP) {
                    if (ph == 1) {
                        if (!swapped) break;
                        lane_row_transpose(x, tb, lane, false);
                    }
                }
                for (uint32_t gi = 0; gi < ngates; gi++) {
                    uint32_t c = s_gc[gi];
                    const bool sw = XP && c - uint32_t(LV) < uint32_t(R);  // lane bits 0..R-1
                    swapped |= sw;
                    if (sw != (ph == 1)) continue;
                    if (sw) c = uint32_t(F) + c - uint32_t(LV);
                    row_gate<R, V, LV, F, false>(x, c, &s_u[gi][(omask >> gi) & 1][0], lane);
                }
            }
            if constexpr (XP) {
                if (swapped) lane_row_transpose(x, tb, lane, true);
            }
        }
        if constexpr (WIN) {
            if (offw1) window(1, offw1);
        }
#pragma unroll
        for (int j = 0; j < NR; j++)
            __stcs(reinterpret_cast<VT *>(rowp + s_off[j]), x[j]);
    }
}

}  // namespace

int row_reg_bits(int elem_bytes, int wide)
{
    if (elem_bytes == 8) return wide ? RowCfg<float2, 1>::R : RowCfg<float2, 0>::R;
    return wide ? RowCfg<double2, 1>::R : RowCfg<double2, 0>::R;
}

int row_fixed_bits(int elem_bytes, int wide)
{
    const int v = elem_bytes == 8 ? (wide ? RowCfg<float2, 1>::V : RowCfg<float2, 0>::V)
                                  : (wide ? RowCfg<double2, 1>::V : RowCfg<double2, 0>::V);
    return 5 + (v == 2 ? 1 : 0);
}

// the shapes the low pass supports: 16 rows of 16 bytes, or (complex64, wide) 32
// rows of 8 bytes
bool row_low_ok(int elem_bytes, int wide) { return elem_bytes == 8 || row_reg_bits(elem_bytes, wide) == 4; }

template <typename E, int W, bool XP, bool REAL, bool WIN>
static cudaError_t launch_row(const uint8_t *dblob, uint64_t poff, uint64_t toff, uint64_t nitems, void *state,
                              int sms, cudaStream_t st)
{
    auto kern = row_pass_kernel<E, W, XP, REAL, WIN>;
    const size_t smem = XP ? size_t(kThreads / 32) * (size_t(1) << RowCfg<E, W>::R) * 32 * sizeof(typename RowCfg<E, W>::VT) : 0;
    if (XP) {
        const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
    }
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
    if (per_sm < 1) per_sm = 1;
    const uint64_t ctas = (nitems + kThreads / 32 - 1) / (kThreads / 32);
    const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ctas, uint64_t(sms) * uint64_t(per_sm))));
    kern<<<grid, kThreads, smem, st>>>(dblob, poff, toff, static_cast<E *>(state));
    return cudaGetLastError();
}

template <typename E, int W, bool XP, bool REAL>
static cudaError_t launch_row_win(const uint8_t *dblob, uint64_t poff, uint64_t toff, uint64_t nitems, bool win,
                                  void *state, int sms, cudaStream_t st)
{
    return win ? launch_row<E, W, XP, REAL, true>(dblob, poff, toff, nitems, state, sms, st)
               : launch_row<E, W, XP, REAL, false>(dblob, poff, toff, nitems, state, sms, st);
}

// The low-pass shapes also run with real gates.
template <typename E, int W>
static cudaError_t launch_row_low(const uint8_t *dblob, uint64_t poff, uint64_t toff, uint64_t nitems, bool low,
                                  bool real, bool win, void *state, int sms, cudaStream_t st)
{
    if (low) return real ? launch_row_win<E, W, true, true>(dblob, poff, toff, nitems, win, state, sms, st)
                         : launch_row_win<E, W, true, false>(dblob, poff, toff, nitems, win, state, sms, st);
    return real ? launch_row_win<E, W, false, true>(dblob, poff, toff, nitems, win, state, sms, st)
                : launch_row_win<E, W, false, false>(dblob, poff, toff, nitems, win, state, sms, st);
}

cudaError_t run_row_pass(const uint8_t *dblob, uint64_t poff, uint64_t toff, uint64_t nitems, int elem_bytes,
                         int wide, bool low, bool real, bool win, void *state, int sms, cudaStream_t st)
{
    // the wide complex64 shape always takes the instance with the window code:
    // ptxas spills far less there (the windows are skipped at run time)
    if (elem_bytes == 8)
        return wide ? launch_row_low<float2, 1>(dblob, poff, toff, nitems, low, real, true, state, sms, st)
                    : launch_row_low<float2, 0>(dblob, poff, toff, nitems, low, real, win, state, sms, st);
    if (wide) return launch_row_low<double2, 1>(dblob, poff, toff, nitems, low, real, win, state, sms, st);
    if (low || real) return cudaErrorInvalidValue;
    return launch_row_win<double2, 0, false, false>(dblob, poff, toff, nitems, win, state, sms, st);
}

}  // namespace zxh
