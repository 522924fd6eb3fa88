// diag.cu -- the diagonal-batch pass (sm_100a): one read-modify-write of the state
// that applies a whole window of commuting p/cp/rz/cz/z gates.
//
// The reference folds a window into six selector buckets and, per amplitude, loops
// over the descriptors of the cross buckets and calls FP64 sin/cos
// (src/zxh/src/kernel/kernel_cuda.cu:505-614, host side :222-344,740-822). Here the
// window is compiled on the host into a polynomial over real-address bits (every
// selector of the benchmark circuits is a single bit after X transport) in 64-bit
// fixed-point turns, so sums wrap exactly modulo 2 pi; multi-bit selectors stay as
// general terms evaluated with parity bit tests on packed masks.
//
// Work split: each WARP owns tiles of 2^T contiguous amplitudes (T = 10 for
// complex64: 16 rows of 64 amplitudes; T = 8 for complex128: 8 rows of 32). A lane
// holds one 16-byte vector per row, all rows loaded before any is used, so every
// warp keeps 4 KB (complex64) in flight with no block-level barrier in the loop.
// Per tile the warp evaluates the tile-dependent coefficients lane-parallel (lane
// k sums the cross terms of tile bit k) and shares them by shuffles; per amplitude
// the phase is two int64 adds (Gray-code walk over rows + a row table) and one
// table-plus-Taylor exp.
#include "core.h"
#include "dev.cuh"
#include "host.h"
#include "sampler.h"

#include <algorithm>
#include <cuda_runtime.h>

namespace zxh {

namespace {

constexpr int kDiagGen = 32;  // general terms handled per window (more are split by the planner)

template <typename E>
struct DiagCfg;
template <>
struct DiagCfg<float2> {
    static constexpr int ROWB = 4;  // log2 rows per warp tile
};
template <>
struct DiagCfg<double2> {
    static constexpr int ROWB = 3;
};

template <typename E>
__global__ void __launch_bounds__(kThreads) diag_kernel(const uint8_t *__restrict__ blob, uint64_t doff, uint64_t toff,
                                                        uint32_t T, uint64_t ntiles, E *__restrict__ state)
{
    using VT = typename ET<E>::VT;
    constexpr int V = ET<E>::V;
    constexpr int LV = (V == 2) ? 1 : 0;
    constexpr int F = 5 + LV;  // lane bits + vector bit
    constexpr int ROWB = DiagCfg<E>::ROWB;
    constexpr int ROWS = 1 << ROWB;
    constexpr int WARPS = kThreads / 32;

    const DiagDev &d = *reinterpret_cast<const DiagDev *>(blob + doff);
    const QuadTerm *iq = reinterpret_cast<const QuadTerm *>(blob + d.off_in_quad);
    const QuadTerm *cr = reinterpret_cast<const QuadTerm *>(blob + d.off_cross);
    const LinTerm *ol = reinterpret_cast<const LinTerm *>(blob + d.off_out_lin);
    const QuadTerm *oq = reinterpret_cast<const QuadTerm *>(blob + d.off_out_quad);
    const GenTerm *gt = reinterpret_cast<const GenTerm *>(blob + d.off_gen);
    const uint32_t *kidx = reinterpret_cast<const uint32_t *>(blob + d.off_kidx);

    __shared__ E s_exp[1 << kExpTableBits];
    __shared__ int64_t s_qi[ROWS];
    __shared__ uint32_t s_gb[WARPS][kDiagGen];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const E *tab = reinterpret_cast<const E *>(blob + toff);
    for (int i = tid; i < (1 << kExpTableBits); i += kThreads) s_exp[i] = tab[i];

    const int IB = int(T) > F ? int(T) - F : 0;
    const int NI = 1 << IB;
    const uint32_t tile_elems = 1u << T;
    const uint32_t ngen = d.n_gen < uint32_t(kDiagGen) ? d.n_gen : uint32_t(kDiagGen);

    // tile-independent parts: quadratic terms inside the tile split into lane-fixed,
    // lane x row, and row-only pieces; linear terms of the lane-fixed bits.
    int64_t qf[V], rho[ROWB][V], linf[V];
#pragma unroll
    for (int v = 0; v < V; v++) {
        qf[v] = 0;
        linf[v] = 0;
#pragma unroll
        for (int l = 0; l < ROWB; l++) rho[l][v] = 0;
    }
    for (uint32_t q = 0; q < d.n_in_quad; q++) {
        const QuadTerm t = iq[q];  // t.i < t.j
#pragma unroll
        for (int v = 0; v < V; v++) {
            const uint32_t e = uint32_t(v) | (uint32_t(lane) << LV);
            const bool bi = int(t.i) < F && ((e >> t.i) & 1);
            if (!bi) continue;
            if (int(t.j) < F) {
                if ((e >> t.j) & 1) qf[v] += t.coef;
            } else {
#pragma unroll
                for (int l = 0; l < ROWB; l++)
                    if (int(t.j) - F == l) rho[l][v] += t.coef;
            }
        }
    }
#pragma unroll
    for (int v = 0; v < V; v++) {
        const uint32_t e = uint32_t(v) | (uint32_t(lane) << LV);
        for (int k = 0; k < F && k < int(T); k++)
            if ((e >> k) & 1) linf[v] += d.lin_in[k];
    }
    if (tid < ROWS) {
        int64_t acc = 0;
        for (uint32_t q = 0; q < d.n_in_quad; q++) {
            const QuadTerm t = iq[q];
            if (int(t.i) >= F && ((tid >> (t.i - F)) & 1) && ((tid >> (t.j - F)) & 1)) acc += t.coef;
        }
        s_qi[tid] = acc;
    }
    __syncthreads();

    const uint64_t stride = uint64_t(gridDim.x) * WARPS;
    for (uint64_t tile = uint64_t(blockIdx.x) * WARPS + uint64_t(warp); tile < ntiles; tile += stride) {
        const uint64_t r = tile << T;  // out-of-tile real bits of this tile
        E *base = state + r;

        // 1. all rows in flight
        VT data[ROWS];
#pragma unroll
        for (int it = 0; it < ROWS; it++) {
            const uint32_t gi = uint32_t(it ^ (it >> 1));
            const uint32_t e0 = (uint32_t(lane) << LV) | (gi << F);
            if (it < NI && e0 < tile_elems) data[it] = __ldcs(reinterpret_cast<const VT *>(base + e0));
        }

        // 2. tile coefficients: lane k < T owns tile bit k; every lane takes a share
        //    of the out-of-tile constant
        int64_t da = 0;
        if (lane < int(T))
            for (uint32_t q = kidx[lane]; q < kidx[lane + 1]; q++) {
                const QuadTerm t = cr[q];
                if ((r >> t.j) & 1) da += t.coef;
            }
        int64_t kp = 0;
        for (uint32_t q = uint32_t(lane); q < d.n_out_lin; q += 32)
            if ((r >> ol[q].bit) & 1) kp += ol[q].coef;
        for (uint32_t q = uint32_t(lane); q < d.n_out_quad; q += 32) {
            const QuadTerm t = oq[q];
            if (((r >> t.i) & 1) && ((r >> t.j) & 1)) kp += t.coef;
        }
        kp = warp_sum_i64(kp) + d.c0;
        if (ngen) {
            for (uint32_t q = uint32_t(lane); q < ngen; q += 32) {
                const GenTerm t = gt[q];
                s_gb[warp][q] = uint32_t(par64(t.a1_out & r) ^ int(t.b1)) | (uint32_t(par64(t.a2_out & r) ^ int(t.b2)) << 1);
            }
            __syncwarp();
        }
        int64_t acc[V], w[ROWB][V];
#pragma unroll
        for (int v = 0; v < V; v++) acc[v] = kp + qf[v] + linf[v];
#pragma unroll
        for (int k = 0; k < F; k++) {
            const int64_t dk = __shfl_sync(0xffffffffu, da, k);
#pragma unroll
            for (int v = 0; v < V; v++) {
                const uint32_t e = uint32_t(v) | (uint32_t(lane) << LV);
                if ((e >> k) & 1) acc[v] += dk;
            }
        }
#pragma unroll
        for (int l = 0; l < ROWB; l++) {
            const int64_t dk = __shfl_sync(0xffffffffu, da, (F + l) & 31);
#pragma unroll
            for (int v = 0; v < V; v++) w[l][v] = (l < IB) ? (d.lin_in[F + l] + dk + rho[l][v]) : 0;
        }

        // 3. rows in Gray-code order: one int64 add per amplitude walks the row bits
#pragma unroll
        for (int it = 0; it < ROWS; it++) {
            const uint32_t gi = uint32_t(it ^ (it >> 1));
            if (it > 0) {
                const int fb = ctz_const(it);
                const bool up = (gi >> fb) & 1;
#pragma unroll
                for (int v = 0; v < V; v++) acc[v] += up ? w[fb][v] : -w[fb][v];
            }
            const uint32_t e0 = (uint32_t(lane) << LV) | (gi << F);
            if (it >= NI || e0 >= tile_elems) continue;
            const int64_t qrow = s_qi[gi];
            VT x = data[it];
#pragma unroll
            for (int v = 0; v < V; v++) {
                int64_t th = acc[v] + qrow;
                const uint32_t e = e0 | uint32_t(v);
                for (uint32_t q = 0; q < ngen; q++) {
                    const uint32_t bb = s_gb[warp][q];
                    const int s1 = par64(gt[q].a1_t & e) ^ int(bb & 1);
                    const int s2 = par64(gt[q].a2_t & e) ^ int(bb >> 1);
                    if (s1 & s2) th += gt[q].coef;
                }
                vset(x, v, cmul(vget(x, v), phase_factor(s_exp, th)));
            }
            __stcs(reinterpret_cast<VT *>(base + e0), x);
        }
        if (ngen) __syncwarp();
    }
}

}  // namespace

cudaError_t run_diag(const uint8_t *dblob, uint64_t doff, uint64_t toff, int m, int elem_bytes, void *state, int sms,
                     cudaStream_t st)
{
    const int Tfull = elem_bytes == 8 ? (6 + DiagCfg<float2>::ROWB) : (5 + DiagCfg<double2>::ROWB);
    const int T = std::min(m, Tfull);
    const uint64_t ntiles = 1ULL << (m - T);
    const uint64_t ctas_needed = (ntiles + kThreads / 32 - 1) / (kThreads / 32);
    int per_sm = 1;
    if (elem_bytes == 8) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, diag_kernel<float2>, kThreads, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, diag_kernel<double2>, kThreads, 0);
    if (per_sm < 1) per_sm = 1;
    const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ctas_needed, uint64_t(sms) * uint64_t(per_sm))));
    if (elem_bytes == 8)
        diag_kernel<float2><<<grid, kThreads, 0, st>>>(dblob, doff, toff, uint32_t(T), ntiles, static_cast<float2 *>(state));
    else
        diag_kernel<double2><<<grid, kThreads, 0, st>>>(dblob, doff, toff, uint32_t(T), ntiles,
                                                        static_cast<double2 *>(state));
    return cudaGetLastError();
}

int diag_tile_bits(int elem_bytes)
{
    return elem_bytes == 8 ? (6 + DiagCfg<float2>::ROWB) : (5 + DiagCfg<double2>::ROWB);
}

}  // namespace zxh
