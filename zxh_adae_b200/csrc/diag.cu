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
// Work split: each WARP owns tiles of 2^T contiguous amplitudes: 2^ROWB rows of 64
// amplitudes (complex64) or 32 (complex128); ROWB is a planner knob, 2 and 3 by
// default (T = 8: 2 KiB and 4 KiB tiles), the fastest on B200 at 26-32 qubits. A lane holds one 16-byte
// vector per row, all rows loaded before any is used, with no block-level barrier
// in the loop.
// A warp takes chunks of 2^cb consecutive tiles and walks each chunk in Gray-code
// order, so from one tile to the next a single out-of-tile bit o flips: the
// tile-dependent coefficients (lane k: the cross sum of tile bit k; the out-of-tile
// constant) move by one entry of dense cross / quadratic tables kept in shared
// memory, and lane l keeps the gradient g_l of the constant with respect to
// out-of-tile bit l. The per-tile cost is then independent of the window's size.
// Per amplitude the phase is two adds (Gray-code walk over rows + a row table) and
// one table-plus-Taylor exp; complex64 does that part in 32-bit turns.
#include "core.h"
#include "dev.cuh"
#include "host.h"
#include "sampler.h"

#include <algorithm>
#include <cuda_runtime.h>

namespace zxh {

namespace {

constexpr int kDiagGen = 32;  // general terms handled per window (more are split by the planner)
constexpr int kDiagOut = 32;  // out-of-tile bits of the incremental walk (2^(32 + T) amplitudes at most)
constexpr int kDiagTileMax = 10;

// FULL: the tile spans all its rows (T = F + ROWB, every state of at least that
// many bits), so no row needs a bounds check.
template <typename E, int ROWB, bool PF, bool FULL>
__global__ void __launch_bounds__(kThreads) diag_kernel(const uint8_t *__restrict__ blob, uint64_t doff, uint64_t toff,
                                                        uint32_t T, uint32_t nout, uint32_t cb, E *__restrict__ state,
                                                        DevStatus *status)
{
    using VT = typename ET<E>::VT;
    constexpr int V = ET<E>::V;
    constexpr int LV = (V == 2) ? 1 : 0;
    constexpr int F = 5 + LV;  // lane bits + vector bit
    constexpr int ROWS = 1 << ROWB;
    constexpr int WARPS = kThreads / 32;

    const DiagDev &d = *reinterpret_cast<const DiagDev *>(blob + doff);
    const QuadTerm *iq = reinterpret_cast<const QuadTerm *>(blob + d.off_in_quad);
    const QuadTerm *cr = reinterpret_cast<const QuadTerm *>(blob + d.off_cross);
    const LinTerm *ol = reinterpret_cast<const LinTerm *>(blob + d.off_out_lin);
    const QuadTerm *oq = reinterpret_cast<const QuadTerm *>(blob + d.off_out_quad);
    const GenTerm *gt = reinterpret_cast<const GenTerm *>(blob + d.off_gen);

    __shared__ E s_exp[1 << kExpTableBits];
    __shared__ int64_t s_qi[ROWS];
    __shared__ uint32_t s_gb[WARPS][kDiagGen];
    __shared__ int64_t s_cross[kDiagTileMax][kDiagOut];  // [tile bit][out bit]
    __shared__ int64_t s_quad[kDiagOut][kDiagOut];       // symmetric, zero diagonal
    __shared__ int64_t s_lin[kDiagOut];
    // complex64: the walk runs in 32-bit turns. Per out bit o: the change of every
    // lane's (and vector slot's) lane-bit phase, of each row weight, and of each
    // out bit's coefficient when bit o flips; and the row-only quadratic parts.
    constexpr int C32 = (V == 2) ? kDiagOut : 1;
    __shared__ uint32_t s_cd32[C32][32][2];           // [out bit][lane][slot]
    __shared__ uint32_t s_cr32[C32][ROWB];            // [out bit][row bit]
    __shared__ uint32_t s_quad32[C32][kDiagOut];      // [out bit][out bit]
    __shared__ uint32_t s_qi32[V == 2 ? ROWS : 1];
    // PF: two tile buffers per warp, filled by TMA bulk copies one tile ahead
    extern __shared__ __align__(128) unsigned char s_tiles[];
    __shared__ __align__(8) uint64_t s_bar[WARPS][2];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const E *tab = reinterpret_cast<const E *>(blob + toff);
    for (int i = tid; i < (1 << kExpTableBits); i += kThreads) s_exp[i] = tab[i];
    for (int i = tid; i < kDiagOut * kDiagOut; i += kThreads) (&s_quad[0][0])[i] = 0;
    for (int i = tid; i < kDiagTileMax * kDiagOut; i += kThreads) (&s_cross[0][0])[i] = 0;
    if (tid < kDiagOut) s_lin[tid] = 0;
    if (PF && tid < WARPS * 2) {
        mbar_init(&s_bar[tid >> 1][tid & 1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    // every (tile bit, out bit), (out bit, out bit) and out bit occurs at most once
    for (uint32_t q = uint32_t(tid); q < d.n_cross; q += kThreads) s_cross[cr[q].i][cr[q].j - T] = cr[q].coef;
    for (uint32_t q = uint32_t(tid); q < d.n_out_quad; q += kThreads) {
        const QuadTerm t = oq[q];
        s_quad[t.i - T][t.j - T] = t.coef;
        s_quad[t.j - T][t.i - T] = t.coef;
    }
    for (uint32_t q = uint32_t(tid); q < d.n_out_lin; q += kThreads) s_lin[ol[q].bit - T] = ol[q].coef;

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
        // branch-free, so qf and rho stay in registers
#pragma unroll
        for (int v = 0; v < V; v++) {
            const uint32_t e = uint32_t(v) | (uint32_t(lane) << LV);
            const int64_t c = (int(t.i) < F && ((e >> t.i) & 1)) ? t.coef : 0;
            qf[v] += (int(t.j) < F && ((e >> t.j) & 1)) ? c : 0;
#pragma unroll
            for (int l = 0; l < ROWB; l++) rho[l][v] += int(t.j) == F + l ? c : 0;
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
        if constexpr (V == 2) s_qi32[tid] = turns32(acc);
    }
    if constexpr (V == 2) {
        __syncthreads();  // s_cross and s_quad are complete
        for (int i = tid; i < kDiagOut * 64; i += kThreads) {
            const int o = i >> 6, l = (i >> 1) & 31, v = i & 1;
            const uint32_t e = uint32_t(v) | (uint32_t(l) << LV);
            int64_t c = 0;
            for (int kk = 0; kk < F && kk < kDiagTileMax; kk++)
                if ((e >> kk) & 1) c += s_cross[kk][o];
            s_cd32[o][l][v] = turns32(c);
        }
        for (int i = tid; i < kDiagOut * ROWB; i += kThreads) {
            const int o = i / ROWB, l = i % ROWB;
            s_cr32[o][l] = F + l < kDiagTileMax ? turns32(s_cross[F + l][o]) : 0u;
        }
        for (int i = tid; i < kDiagOut * kDiagOut; i += kThreads) (&s_quad32[0][0])[i] = turns32((&s_quad[0][0])[i]);
    }
    __syncthreads();

    const uint64_t nchunks = 1ULL << (nout - cb);
    const uint64_t stride = uint64_t(gridDim.x) * WARPS;
    const uint32_t tile_bytes = uint32_t(sizeof(E)) << T;
    E *tbuf = reinterpret_cast<E *>(s_tiles) + size_t(warp) * 2 * tile_elems;
    uint32_t k = 0;  // tiles this warp has taken
    if (PF && lane == 0 && uint64_t(blockIdx.x) * WARPS + uint64_t(warp) < nchunks) {
        const uint64_t t = (uint64_t(blockIdx.x) * WARPS + uint64_t(warp)) << cb;
        mbar_arrive_expect_tx(&s_bar[warp][0], tile_bytes);
        bulk_g2s(tbuf, state + (t << T), tile_bytes, &s_bar[warp][0]);
    }
    for (uint64_t chunk = uint64_t(blockIdx.x) * WARPS + uint64_t(warp); chunk < nchunks; chunk += stride) {
        const uint64_t t0 = chunk << cb;
        // coefficients of the chunk's first tile, from the dense tables
        int64_t da = 0, g = 0, h = 0;
        if (lane < int(T))
            for (uint32_t o = 0; o < nout; o++)
                if ((t0 >> o) & 1) da += s_cross[lane][o];
        if (lane < int(nout)) {
            g = s_lin[lane];
            for (uint32_t o = 0; o < nout; o++)
                if ((t0 >> o) & 1) {
                    g += s_quad[lane][o];
                    if (int(o) < lane) h += s_quad[lane][o];
                }
            h = ((t0 >> lane) & 1) ? h + s_lin[lane] : 0;
        }
        int64_t kp = warp_sum_i64(h) + d.c0;
        // complex64: the walk state in 32-bit turns, updated per tile from the
        // shared 32-bit tables (no shuffles of 64-bit coefficients per tile): kp32
        // the out-bit part, g32 this lane's out-bit coefficient, lp32 this lane's
        // lane-bit part (both vector slots, with its tile-constant terms), w32 the
        // row weights
        [[maybe_unused]] uint32_t kp32 = 0, g32 = 0, lp32[V], w32[ROWB][V];
        if constexpr (V == 2) {
            kp32 = turns32(kp);
            g32 = turns32(g);
            int64_t lp[V];
#pragma unroll
            for (int v = 0; v < V; v++) lp[v] = qf[v] + linf[v];
#pragma unroll
            for (int kk = 0; kk < F; kk++) {
                const int64_t dk = __shfl_sync(0xffffffffu, da, kk);
#pragma unroll
                for (int v = 0; v < V; v++) {
                    const uint32_t e = uint32_t(v) | (uint32_t(lane) << LV);
                    if ((e >> kk) & 1) lp[v] += dk;
                }
            }
#pragma unroll
            for (int v = 0; v < V; v++) lp32[v] = turns32(lp[v]);
#pragma unroll
            for (int l = 0; l < ROWB; l++) {
                const int64_t dk = __shfl_sync(0xffffffffu, da, (F + l) & 31);
#pragma unroll
                for (int v = 0; v < V; v++) w32[l][v] = (l < IB) ? turns32(d.lin_in[F + l] + dk + rho[l][v]) : 0u;
            }
        }

    for (uint32_t it_t = 0; it_t < (1u << cb); it_t++, k++) {
        const uint64_t tile = t0 | uint64_t(it_t ^ (it_t >> 1));
        const uint64_t r = tile << T;  // out-of-tile real bits of this tile
        E *base = state + r;

        // 1. all rows in flight. PF: the tile is in shared memory (or on its way);
        //    once it has landed, start the copy of the next one into the other
        //    buffer, last read by the previous tile (whose values every lane has
        //    consumed). The warp gives up as one; then only this tile's copy can
        //    still be in flight, and it waits for that (bounded) before leaving.
        const E *src = base;
        if constexpr (PF) {
            __syncwarp();
            if (!__all_sync(0xffffffffu, mbar_wait_bounded(&s_bar[warp][k & 1], (k >> 1) & 1))) {
                if (lane == 0) report(status, kErrTimeout, 7, tile);
                (void)mbar_wait_bounded(&s_bar[warp][k & 1], (k >> 1) & 1);
                return;
            }
            uint64_t nt = 0;
            bool has = true;
            if (it_t + 1 < (1u << cb)) nt = t0 | uint64_t((it_t + 1) ^ ((it_t + 1) >> 1));
            else if (chunk + stride < nchunks) nt = (chunk + stride) << cb;
            else has = false;
            if (has && lane == 0) {
                uint64_t *nb = &s_bar[warp][(k + 1) & 1];
                mbar_arrive_expect_tx(nb, tile_bytes);
                bulk_g2s(tbuf + size_t((k + 1) & 1) * tile_elems, state + (nt << T), tile_bytes, nb);
            }
            src = tbuf + size_t(k & 1) * tile_elems;
        }
        VT data[ROWS];
#pragma unroll
        for (int it = 0; it < ROWS; it++) {
            const uint32_t gi = uint32_t(it ^ (it >> 1));
            const uint32_t e0 = (uint32_t(lane) << LV) | (gi << F);
            if (FULL || (it < NI && e0 < tile_elems)) {
                if constexpr (PF) data[it] = *reinterpret_cast<const VT *>(src + e0);
                else data[it] = __ldcs(reinterpret_cast<const VT *>(src + e0));
            }
        }

        // 2. one out-of-tile bit o flipped since the previous tile of the chunk
        if (it_t > 0) {
            const int o = __ffs(it_t) - 1;
            const bool up = (tile >> o) & 1;
            if constexpr (V == 2) {
                const uint32_t go = __shfl_sync(0xffffffffu, g32, o);
                kp32 += up ? go : 0u - go;
                const uint32_t dq = s_quad32[o][lane];  // zero for lanes past the out bits
                g32 += up ? dq : 0u - dq;
                const uint2 dc = *reinterpret_cast<const uint2 *>(&s_cd32[o][lane][0]);
                lp32[0] += up ? dc.x : 0u - dc.x;
                lp32[1] += up ? dc.y : 0u - dc.y;
#pragma unroll
                for (int l = 0; l < ROWB; l++) {
                    const uint32_t dr = s_cr32[o][l];  // zero for row bits outside the tile
#pragma unroll
                    for (int v = 0; v < V; v++) w32[l][v] += up ? dr : 0u - dr;
                }
            } else {
                const int64_t go = __shfl_sync(0xffffffffu, g, o);
                kp += up ? go : -go;
                if (lane < int(nout)) g += up ? s_quad[o][lane] : -s_quad[o][lane];
                if (lane < int(T)) da += up ? s_cross[lane][o] : -s_cross[lane][o];
            }
        }
        if (ngen) {
            for (uint32_t q = uint32_t(lane); q < ngen; q += 32) {
                const GenTerm t = gt[q];
                s_gb[warp][q] = uint32_t(par64(t.a1_out & r) ^ int(t.b1)) | (uint32_t(par64(t.a2_out & r) ^ int(t.b2)) << 1);
            }
            __syncwarp();
        }
        // 3. rows in Gray-code order: one add per amplitude walks the row bits.
        //    complex64 carries the per-amplitude phase in 32-bit turns (2 pi / 2^32
        //    resolution; every coefficient is rounded once to that grid, so a phase
        //    is off by at most half a step per term it sums).
        if constexpr (V == 2) {
            uint32_t a32[V];
#pragma unroll
            for (int v = 0; v < V; v++) a32[v] = kp32 + lp32[v];
#pragma unroll
            for (int it = 0; it < ROWS; it++) {
                const uint32_t gi = uint32_t(it ^ (it >> 1));
                if (it > 0) {
                    const int fb = ctz_const(it);
                    const bool up = (gi >> fb) & 1;
#pragma unroll
                    for (int v = 0; v < V; v++) a32[v] += up ? w32[fb][v] : 0u - w32[fb][v];
                }
                const uint32_t e0 = (uint32_t(lane) << LV) | (gi << F);
                if (!FULL && (it >= NI || e0 >= tile_elems)) continue;
                const uint32_t qrow = s_qi32[gi];
                VT x = data[it];
                uint32_t th[V];
#pragma unroll
                for (int v = 0; v < V; v++) th[v] = a32[v] + qrow;
                if (ngen) {
#pragma unroll
                    for (int v = 0; v < V; v++) {
                        const uint32_t e = e0 | uint32_t(v);
                        for (uint32_t q = 0; q < ngen; q++) {
                            const uint32_t bb = s_gb[warp][q];
                            const int s1 = par64(gt[q].a1_t & e) ^ int(bb & 1);
                            const int s2 = par64(gt[q].a2_t & e) ^ int(bb >> 1);
                            if (s1 & s2) th[v] += turns32(gt[q].coef);
                        }
                    }
                }
#pragma unroll
                for (int v = 0; v < V; v++)
                    vset(x, v, cmul(vget(x, v), phase_factor32(reinterpret_cast<const float2 *>(s_exp), th[v])));
                __stcs(reinterpret_cast<VT *>(base + e0), x);
            }
        } else {
        int64_t acc[V], w[ROWB][V];
#pragma unroll
        for (int v = 0; v < V; v++) acc[v] = kp + qf[v] + linf[v];
#pragma unroll
        for (int kk = 0; kk < F; kk++) {
            const int64_t dk = __shfl_sync(0xffffffffu, da, kk);
#pragma unroll
            for (int v = 0; v < V; v++) {
                const uint32_t e = uint32_t(v) | (uint32_t(lane) << LV);
                if ((e >> kk) & 1) acc[v] += dk;
            }
        }
#pragma unroll
        for (int l = 0; l < ROWB; l++) {
            const int64_t dk = __shfl_sync(0xffffffffu, da, (F + l) & 31);
#pragma unroll
            for (int v = 0; v < V; v++) w[l][v] = (l < IB) ? (d.lin_in[F + l] + dk + rho[l][v]) : 0;
        }
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
            if (!FULL && (it >= NI || e0 >= tile_elems)) continue;
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
        }
        if (ngen) __syncwarp();
    }
    }
}

}  // namespace

namespace {

template <typename E, int ROWB, bool PF, bool FULL>
cudaError_t launch_diag(const uint8_t *dblob, uint64_t doff, uint64_t toff, int m, int chunk_bits, E *state,
                        DevStatus *status, int sms, cudaStream_t st)
{
    const int Tfull = (ET<E>::V == 2 ? 6 : 5) + ROWB;
    const int T = std::min(m, Tfull);
    const int nout = m - T;
    if (nout > kDiagOut) return cudaErrorInvalidValue;
    auto kern = diag_kernel<E, ROWB, PF, FULL>;
    const size_t smem = PF ? size_t(kThreads / 32) * 2 * (sizeof(E) << T) : 0;
    if (PF) {
        const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
    }
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
    if (per_sm < 1) per_sm = 1;
    // chunks of 2^cb tiles: a chunk spans 32 KiB (16 complex64 tiles of 2 KiB, 8
    // complex128 tiles of 4 KiB at the default row counts), the fastest on B200 at
    // 26-32 qubits
    int cb = chunk_bits;
    if (cb < 0) {
        cb = 0;
        while ((size_t(sizeof(E)) << (T + cb)) < (size_t(32) << 10)) cb++;
    }
    cb = std::min(cb, nout);
    const uint64_t nchunks = 1ULL << (nout - cb);
    const uint64_t ctas_needed = (nchunks + kThreads / 32 - 1) / (kThreads / 32);
    const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ctas_needed, uint64_t(sms) * uint64_t(per_sm))));
    kern<<<grid, kThreads, smem, st>>>(dblob, doff, toff, uint32_t(T), uint32_t(nout), uint32_t(cb), state, status);
    return cudaGetLastError();
}

template <typename E, int ROWB>
cudaError_t launch_diag_pf(const uint8_t *dblob, uint64_t doff, uint64_t toff, int m, int chunk_bits, bool pf,
                           E *state, DevStatus *status, int sms, cudaStream_t st)
{
    const bool full = m >= (ET<E>::V == 2 ? 6 : 5) + ROWB;
    if (full)
        return pf ? launch_diag<E, ROWB, true, true>(dblob, doff, toff, m, chunk_bits, state, status, sms, st)
                  : launch_diag<E, ROWB, false, true>(dblob, doff, toff, m, chunk_bits, state, status, sms, st);
    return pf ? launch_diag<E, ROWB, true, false>(dblob, doff, toff, m, chunk_bits, state, status, sms, st)
              : launch_diag<E, ROWB, false, false>(dblob, doff, toff, m, chunk_bits, state, status, sms, st);
}

}  // namespace

cudaError_t run_diag(const uint8_t *dblob, uint64_t doff, uint64_t toff, int m, int elem_bytes, int row_bits,
                     int chunk_bits, bool prefetch, void *state, DevStatus *status, int sms, cudaStream_t st)
{
    if (elem_bytes == 8) {
        auto *s = static_cast<float2 *>(state);
        switch (row_bits) {
        case 2: return launch_diag_pf<float2, 2>(dblob, doff, toff, m, chunk_bits, prefetch, s, status, sms, st);
        case 3: return launch_diag_pf<float2, 3>(dblob, doff, toff, m, chunk_bits, prefetch, s, status, sms, st);
        case 4: return launch_diag_pf<float2, 4>(dblob, doff, toff, m, chunk_bits, prefetch, s, status, sms, st);
        default: return cudaErrorInvalidValue;
        }
    }
    auto *s = static_cast<double2 *>(state);
    switch (row_bits) {
    case 2: return launch_diag_pf<double2, 2>(dblob, doff, toff, m, chunk_bits, prefetch, s, status, sms, st);
    case 3: return launch_diag_pf<double2, 3>(dblob, doff, toff, m, chunk_bits, prefetch, s, status, sms, st);
    case 4: return launch_diag_pf<double2, 4>(dblob, doff, toff, m, chunk_bits, prefetch, s, status, sms, st);
    default: return cudaErrorInvalidValue;
    }
}

int diag_tile_bits(int elem_bytes, int row_bits) { return (elem_bytes == 8 ? 6 : 5) + row_bits; }

}  // namespace zxh
