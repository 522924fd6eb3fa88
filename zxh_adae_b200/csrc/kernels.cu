// kernels.cu -- sm_100a state-vector kernels of the B200-native ZXH path.
//
//   product_kernel  writes a product state in one pass (the reference applies each
//                   first-touch H/U3 as its own sweep over a growing state,
//                   zxh.cpp:782-825 + kernel_cuda.cu:346-361).
//   expand_kernel   one lazy-expansion step, 2^m -> 2^(m+1) amplitudes, fused with
//                   the pair op that caused it (sv_common.cpp:330-349).
//   tile_kernel     the U3-batch / diagonal-batch pass: TMA bulk-copies a tile of
//                   2^T amplitudes (2^c contiguous x 2^h strided chunks) into shared
//                   memory, applies every queued step there (diagonal windows with
//                   phases from bit tests on packed masks, 2x2 pair ops), and bulk-
//                   stores it back once. Replaces u3_block_batch_kernel_cuda (one grid
//                   sweep per descriptor, kernel_cuda.cu:390-423) and
//                   diag_block_kernel_cuda (kernel_cuda.cu:505-614).
//   scatter_kernel  get_state: real -> virtual index, bit reversal, global phase
//                   (zxh.cpp:579-636).
#include "core.h"
#include "dev.cuh"
#include "host.h"
#include "sampler.h"

#include <algorithm>

#include <cuda_runtime.h>

namespace zxh {

// ---------------------------------------------------------------------------
// product state

template <typename E>
__global__ void __launch_bounds__(kThreads) product_kernel(const uint8_t *__restrict__ blob, uint64_t off,
                                                           uint64_t tab_off, E *__restrict__ state)
{
    using VT = typename ET<E>::VT;
    constexpr int V = ET<E>::V;
    const ProductDev p = *reinterpret_cast<const ProductDev *>(blob + off);
    const E *L = reinterpret_cast<const E *>(blob + tab_off);
    const E *M = L + (1u << p.c0);
    const E *H = M + (1u << p.c1);
    const uint64_t n = 1ULL << p.m;
    const uint64_t m0 = (1ULL << p.c0) - 1, m1 = (1ULL << p.c1) - 1;
    const uint32_t s1 = p.c0, s2 = p.c0 + p.c1;
    if (n < uint64_t(V)) {  // a single complex64 amplitude
        if (blockIdx.x == 0 && threadIdx.x == 0) state[0] = cmul(cmul(L[0], M[0]), H[0]);
        return;
    }
    const uint64_t nv = n / V;
    for (uint64_t i = uint64_t(blockIdx.x) * kThreads + threadIdx.x; i < nv; i += uint64_t(gridDim.x) * kThreads) {
        VT x;
#pragma unroll
        for (int v = 0; v < V; v++) {
            const uint64_t y = i * V + v;
            vset(x, v, cmul(cmul(__ldg(&L[y & m0]), __ldg(&M[(y >> s1) & m1])), __ldg(&H[y >> s2])));
        }
        __stcs(reinterpret_cast<VT *>(state) + i, x);
    }
}

// ---------------------------------------------------------------------------
// lazy expansion fused with its pair op

template <typename E>
__global__ void __launch_bounds__(kThreads) expand_kernel(const uint8_t *__restrict__ blob, uint64_t off,
                                                          E *__restrict__ state)
{
    using R = typename ET<E>::R;
    const ExpandDev *p = reinterpret_cast<const ExpandDev *>(blob + off);
    const uint64_t half = 1ULL << p->m_old;
    const uint64_t alpha = p->alpha, calpha = p->ctrl_alpha;
    const int beta = int(p->beta), cbeta = int(p->ctrl_beta), has_ctrl = int(p->has_ctrl);
    const R u00r = R(p->u[0]), u00i = R(p->u[1]), u01r = R(p->u[2]), u01i = R(p->u[3]);
    const R u10r = R(p->u[4]), u10i = R(p->u[5]), u11r = R(p->u[6]), u11i = R(p->u[7]);
    for (uint64_t i = uint64_t(blockIdx.x) * kThreads + threadIdx.x; i < half; i += uint64_t(gridDim.x) * kThreads) {
        const E a = state[i];
        const int s = par64(i & alpha) ^ beta;
        const bool on = !has_ctrl || (par64(i & calpha) ^ cbeta);
        E lo, hi;
        if (!on) {
            lo = a;
            hi.x = R(0);
            hi.y = R(0);
        } else if (!s) {  // i even: new[i] = u00 a, new[i+half] = u10 a
            lo.x = u00r * a.x - u00i * a.y;
            lo.y = u00r * a.y + u00i * a.x;
            hi.x = u10r * a.x - u10i * a.y;
            hi.y = u10r * a.y + u10i * a.x;
        } else {  // i odd: new[i] = u11 a, new[i+half] = u01 a
            lo.x = u11r * a.x - u11i * a.y;
            lo.y = u11r * a.y + u11i * a.x;
            hi.x = u01r * a.x - u01i * a.y;
            hi.y = u01r * a.y + u01i * a.x;
        }
        state[i] = lo;
        state[i + half] = hi;
    }
}

// ---------------------------------------------------------------------------
// pair op straight in global memory

template <typename E>
__global__ void __launch_bounds__(kThreads) pair_kernel(const uint8_t *__restrict__ blob, uint64_t off,
                                                        E *__restrict__ state)
{
    using R = typename ET<E>::R;
    const PairDev *p = reinterpret_cast<const PairDev *>(blob + off);
    const uint64_t npairs = 1ULL << (p->m - 1);
    const uint32_t pv = p->pivot;
    const uint64_t delta = p->delta, alpha = p->alpha, calpha = p->ctrl_alpha;
    const int beta = int(p->beta), cbeta = int(p->ctrl_beta), has_ctrl = int(p->has_ctrl);
    const R u00r = R(p->u[0]), u00i = R(p->u[1]), u01r = R(p->u[2]), u01i = R(p->u[3]);
    const R u10r = R(p->u[4]), u10i = R(p->u[5]), u11r = R(p->u[6]), u11i = R(p->u[7]);
    for (uint64_t q = uint64_t(blockIdx.x) * kThreads + threadIdx.x; q < npairs; q += uint64_t(gridDim.x) * kThreads) {
        uint64_t e0 = ((q >> pv) << (pv + 1)) | (q & ((1ULL << pv) - 1ULL));
        uint64_t e1 = e0 ^ delta;
        if (par64(alpha & e0) ^ beta) {
            const uint64_t t = e0;
            e0 = e1;
            e1 = t;
        }
        if (has_ctrl && !(par64(calpha & e0) ^ cbeta)) continue;
        const E a = state[e0], b = state[e1];
        E x, y;
        x.x = u00r * a.x - u00i * a.y + u01r * b.x - u01i * b.y;
        x.y = u00r * a.y + u00i * a.x + u01r * b.y + u01i * b.x;
        y.x = u10r * a.x - u10i * a.y + u11r * b.x - u11i * b.y;
        y.y = u10r * a.y + u10i * a.x + u11r * b.y + u11i * b.x;
        state[e0] = x;
        state[e1] = y;
    }
}

// ---------------------------------------------------------------------------
// tile pass

constexpr int kMaxDiag = 2;     // diagonal windows per tile pass (prologue + epilogue)
constexpr int kMaxGen = 64;     // general (multi-bit selector) terms per window
constexpr int kIterBits = 4;    // tile bits above the per-thread fixed bits

template <typename E>
struct TileSmem {
    uint64_t mbar[2];
    uint64_t r[2];
    int64_t da[kMaxDiag][kMaxTileBits];
    int64_t K[kMaxDiag];
    int64_t qi[kMaxDiag][1 << kIterBits];
    uint32_t gb[kMaxDiag][kMaxGen];
    uint32_t ub[64];
};

__device__ __forceinline__ uint64_t pdep64(uint64_t x, uint64_t mask)
{
    uint64_t r = 0;
    for (uint64_t bb = 1; mask; bb += bb) {
        const uint64_t low = mask & (0 - mask);
        if (x & bb) r |= low;
        mask &= mask - 1;
    }
    return r;
}

__device__ __forceinline__ uint64_t chunk_base(const TileDev &g, uint64_t r, uint32_t j)
{
    uint64_t a = r;
    for (uint32_t b = 0; b < g.h; b++)
        if ((j >> b) & 1) a |= 1ULL << g.pos[g.c + b];
    return a;
}

// Issues the bulk copies of one tile (warp 0 only).
template <typename E>
__device__ __forceinline__ void issue_tile_load(const TileDev &g, const E *state, E *buf, uint64_t r, uint64_t *bar,
                                                int lane)
{
    const uint32_t nchunk = 1u << g.h;
    const uint32_t cbytes = uint32_t(sizeof(E)) << g.c;
    if (lane == 0) mbar_arrive_expect_tx(bar, cbytes * nchunk);
    __syncwarp();
    for (uint32_t j = uint32_t(lane); j < nchunk; j += 32)
        bulk_g2s(buf + (size_t(j) << g.c), state + chunk_base(g, r, j), cbytes, bar);
}

template <typename E>
__device__ __forceinline__ void issue_tile_store(const TileDev &g, E *state, const E *buf, uint64_t r, int lane)
{
    const uint32_t nchunk = 1u << g.h;
    const uint32_t cbytes = uint32_t(sizeof(E)) << g.c;
    for (uint32_t j = uint32_t(lane); j < nchunk; j += 32)
        bulk_s2g(state + chunk_base(g, r, j), buf + (size_t(j) << g.c), cbytes);
    bulk_commit();
}

template <typename E>
__global__ void __launch_bounds__(kThreads) tile_kernel(const uint8_t *__restrict__ blob, uint64_t goff,
                                                        E *__restrict__ state, DevStatus *status)
{
    using R = typename ET<E>::R;
    constexpr int V = ET<E>::V;
    constexpr int LV = (V == 2) ? 1 : 0;
    constexpr int F = 8 + LV;  // fixed bits of a thread's elements: vector lane + thread index

    const TileDev g = *reinterpret_cast<const TileDev *>(blob + goff);
    const StepDev *steps = reinterpret_cast<const StepDev *>(blob + g.off_steps);
    extern __shared__ __align__(128) unsigned char dsm[];
    __shared__ TileSmem<E> S;
    const uint32_t T = g.T;
    const uint32_t tile_elems = 1u << T;
    E *bufs[2] = {reinterpret_cast<E *>(dsm), reinterpret_cast<E *>(dsm) + tile_elems};
    const int tid = int(threadIdx.x), lane = tid & 31, warp = tid >> 5;
    const uint32_t nsteps = g.nsteps;
    const int IB = int(T) > F ? int(T) - F : 0;  // iteration bits
    const int NI = 1 << IB;

    // ---- tile-independent per-thread precompute of the diagonal windows ----
    int64_t qf[kMaxDiag][V];
    int64_t rho[kMaxDiag][kIterBits][V];
    int ndiag = 0;
    for (uint32_t si = 0; si < nsteps; si++) {
        if (steps[si].kind != STEP_DIAG || ndiag >= kMaxDiag) continue;
        const DiagDev &d = *reinterpret_cast<const DiagDev *>(blob + steps[si].off);
        const QuadTerm *iq = reinterpret_cast<const QuadTerm *>(blob + d.off_in_quad);
#pragma unroll
        for (int v = 0; v < V; v++) {
            qf[ndiag][v] = 0;
#pragma unroll
            for (int l = 0; l < kIterBits; l++) rho[ndiag][l][v] = 0;
        }
        for (uint32_t q = 0; q < d.n_in_quad; q++) {
            const QuadTerm t = iq[q];  // t.i < t.j (tile coordinates)
#pragma unroll
            for (int v = 0; v < V; v++) {
                const uint32_t e = uint32_t(v) | (uint32_t(tid) << LV);
                const int bi = int(t.i) < F ? int((e >> t.i) & 1) : -1;
                const int bj = int(t.j) < F ? int((e >> t.j) & 1) : -1;
                if (bi == 1 && bj == 1) qf[ndiag][v] += t.coef;
                else if (bi == 1 && bj < 0) rho[ndiag][t.j - F][v] += t.coef;
            }
        }
        if (tid < NI) {
            int64_t acc = 0;
            for (uint32_t q = 0; q < d.n_in_quad; q++) {
                const QuadTerm t = iq[q];
                if (int(t.i) >= F && ((tid >> (t.i - F)) & 1) && ((tid >> (t.j - F)) & 1)) acc += t.coef;
            }
            S.qi[ndiag][tid] = acc;
        }
        ndiag++;
    }

    if (tid == 0) {
        mbar_init(&S.mbar[0], 1);
        mbar_init(&S.mbar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();

    uint64_t tidx = blockIdx.x;
    if (tidx >= g.ntiles) return;
    // Chunks below 16 bytes cannot be bulk-copied: such tiny states are moved with
    // plain loads and stores (only a 1-amplitude complex64 state gets here).
    const bool direct = (uint32_t(sizeof(E)) << g.c) < 16u;
    if (direct) {
        if (tid == 0) S.r[0] = pdep64(tidx, g.free_mask);
        __syncthreads();
        for (uint32_t e = uint32_t(tid); e < tile_elems; e += kThreads)
            bufs[0][e] = state[chunk_base(g, S.r[0], e >> g.c) + (e & ((1u << g.c) - 1u))];
        __syncthreads();
    } else if (warp == 0) {
        uint64_t r0 = 0;
        if (lane == 0) {
            r0 = pdep64(tidx, g.free_mask);
            S.r[0] = r0;
        }
        r0 = __shfl_sync(0xffffffffu, r0, 0);
        issue_tile_load(g, state, bufs[0], r0, &S.mbar[0], lane);
    }

    for (uint32_t k = 0;; k++, tidx += gridDim.x) {
        if (tidx >= g.ntiles) break;
        const int s = int(k & 1);
        const uint64_t nxt = tidx + gridDim.x;
        if (!direct && warp == 0 && nxt < g.ntiles) {
            bulk_wait_read0();  // stores of the tile that used the other stage have read it
            __syncwarp();
            uint64_t rn = 0;
            if (lane == 0) {
                rn = pdep64(nxt, g.free_mask);
                S.r[s ^ 1] = rn;
            }
            rn = __shfl_sync(0xffffffffu, rn, 0);
            issue_tile_load(g, state, bufs[s ^ 1], rn, &S.mbar[s ^ 1], lane);
        }
        if (direct) {
            if (k > 0) {
                if (tid == 0) S.r[s] = pdep64(tidx, g.free_mask);
                __syncthreads();
                for (uint32_t e = uint32_t(tid); e < tile_elems; e += kThreads)
                    bufs[s][e] = state[chunk_base(g, S.r[s], e >> g.c) + (e & ((1u << g.c) - 1u))];
                __syncthreads();
            }
        } else if (__syncthreads_or(!mbar_wait_bounded(&S.mbar[s], (k >> 1) & 1))) {
            // the block gives up as one; this tile's copy and the next one's (issued
            // above) may still be in flight: wait for both, bounded, before leaving
            if (tid == 0) report(status, kErrTimeout, 1, tidx);
            (void)mbar_wait_bounded(&S.mbar[s], (k >> 1) & 1);
            if (nxt < g.ntiles) (void)mbar_wait_bounded(&S.mbar[s ^ 1], ((k + 1) >> 1) & 1);
            if (warp == 0) bulk_wait0();
            return;
        }
        E *buf = bufs[s];
        const uint64_t r = S.r[s];

        // ---- per-tile parameters ----
        for (int d = 0; d < ndiag; d++) {
            if (tid < kMaxTileBits) S.da[d][tid] = 0;
            if (tid == 0) S.K[d] = 0;
        }
        __syncthreads();
        {
            int d = 0;
            for (uint32_t si = 0; si < nsteps; si++) {
                const StepDev st = steps[si];
                if (st.kind == STEP_U3) {
                    if (tid == 0) {
                        const U3Dev &u = *reinterpret_cast<const U3Dev *>(blob + st.off);
                        S.ub[si & 63] = uint32_t(par64(u.alpha_out & r) ^ int(u.beta)) |
                                        (uint32_t(par64(u.ctrl_out & r) ^ int(u.ctrl_beta)) << 1);
                    }
                    continue;
                }
                if (d >= kMaxDiag) continue;
                const DiagDev &dd = *reinterpret_cast<const DiagDev *>(blob + st.off);
                const QuadTerm *cr = reinterpret_cast<const QuadTerm *>(blob + dd.off_cross);
                const LinTerm *ol = reinterpret_cast<const LinTerm *>(blob + dd.off_out_lin);
                const QuadTerm *oq = reinterpret_cast<const QuadTerm *>(blob + dd.off_out_quad);
                const GenTerm *gt = reinterpret_cast<const GenTerm *>(blob + dd.off_gen);
                int64_t kacc = 0;
                for (uint32_t q = uint32_t(tid); q < dd.n_cross; q += kThreads) {
                    const QuadTerm t = cr[q];
                    if ((r >> t.j) & 1) atomicAdd(reinterpret_cast<unsigned long long *>(&S.da[d][t.i]),
                                                  static_cast<unsigned long long>(t.coef));
                }
                for (uint32_t q = uint32_t(tid); q < dd.n_out_lin; q += kThreads)
                    if ((r >> ol[q].bit) & 1) kacc += ol[q].coef;
                for (uint32_t q = uint32_t(tid); q < dd.n_out_quad; q += kThreads)
                    if (((r >> oq[q].i) & 1) && ((r >> oq[q].j) & 1)) kacc += oq[q].coef;
                kacc = warp_sum_i64(kacc);
                if (lane == 0 && kacc != 0)
                    atomicAdd(reinterpret_cast<unsigned long long *>(&S.K[d]), static_cast<unsigned long long>(kacc));
                for (uint32_t q = uint32_t(tid); q < dd.n_gen && q < uint32_t(kMaxGen); q += kThreads) {
                    const GenTerm t = gt[q];
                    S.gb[d][q] = uint32_t(par64(t.a1_out & r) ^ int(t.b1)) | (uint32_t(par64(t.a2_out & r) ^ int(t.b2)) << 1);
                }
                d++;
            }
        }
        __syncthreads();

        // ---- steps ----
        int d = 0;
        for (uint32_t si = 0; si < nsteps; si++) {
            const StepDev st = steps[si];
            if (st.kind == STEP_DIAG) {
                if (d >= kMaxDiag) continue;
                const DiagDev &dd = *reinterpret_cast<const DiagDev *>(blob + st.off);
                const GenTerm *gt = reinterpret_cast<const GenTerm *>(blob + dd.off_gen);
                const uint32_t ngen = dd.n_gen < uint32_t(kMaxGen) ? dd.n_gen : uint32_t(kMaxGen);
                const int64_t K = S.K[d] + dd.c0;
                int64_t acc[V];
                int64_t w[kIterBits][V];
#pragma unroll
                for (int v = 0; v < V; v++) {
                    const uint32_t e = uint32_t(v) | (uint32_t(tid) << LV);
                    int64_t a = K + qf[d][v];
                    for (int kb = 0; kb < F && kb < int(T); kb++)
                        if ((e >> kb) & 1) a += dd.lin_in[kb] + S.da[d][kb];
                    acc[v] = a;
#pragma unroll
                    for (int l = 0; l < kIterBits; l++)
                        w[l][v] = (l < IB) ? (dd.lin_in[F + l] + S.da[d][F + l] + rho[d][l][v]) : 0;
                }
                for (int it = 0; it < NI; it++) {
                    const int gi = it ^ (it >> 1);
                    if (it > 0) {
                        const int fb = __ffs(it) - 1;
                        const bool set = (gi >> fb) & 1;
#pragma unroll
                        for (int l = 0; l < kIterBits; l++)
                            if (l == fb) {
#pragma unroll
                                for (int v = 0; v < V; v++) acc[v] += set ? w[l][v] : -w[l][v];
                            }
                    }
                    const uint32_t e0 = (uint32_t(tid) << LV) | (uint32_t(gi) << F);
                    if (e0 >= tile_elems) continue;
                    const int64_t qi = S.qi[d][gi];
#pragma unroll
                    for (int v = 0; v < V; v++) {
                        const uint32_t e = e0 | uint32_t(v);
                        if (e >= tile_elems) continue;
                        int64_t th = acc[v] + qi;
                        for (uint32_t q = 0; q < ngen; q++) {
                            const uint32_t bb = S.gb[d][q];
                            const int s1 = par64(gt[q].a1_t & e) ^ int(bb & 1);
                            const int s2 = par64(gt[q].a2_t & e) ^ int(bb >> 1);
                            if (s1 & s2) th += gt[q].coef;
                        }
                        buf[e] = apply_phase(buf[e], th);
                    }
                }
                d++;
            } else {
                const U3Dev &u = *reinterpret_cast<const U3Dev *>(blob + st.off);
                const uint32_t ub = S.ub[si & 63];
                const int beta = int(ub & 1), cbeta = int(ub >> 1);
                const uint64_t dt = u.delta_t, at = u.alpha_t, ct = u.ctrl_t;
                const uint32_t pv = u.pivot;
                const int has_ctrl = int(u.has_ctrl);
                const R u00r = R(u.u[0]), u00i = R(u.u[1]), u01r = R(u.u[2]), u01i = R(u.u[3]);
                const R u10r = R(u.u[4]), u10i = R(u.u[5]), u11r = R(u.u[6]), u11i = R(u.u[7]);
                const uint32_t npairs = tile_elems >> 1;
                for (uint32_t p = uint32_t(tid); p < npairs; p += kThreads) {
                    uint32_t e0 = ((p >> pv) << (pv + 1)) | (p & ((1u << pv) - 1u));
                    uint32_t e1 = e0 ^ uint32_t(dt);
                    if (par64(at & e0) ^ beta) {
                        const uint32_t t = e0;
                        e0 = e1;
                        e1 = t;
                    }
                    if (has_ctrl && !(par64(ct & e0) ^ cbeta)) continue;
                    const E a = buf[e0], b = buf[e1];
                    E x, y;
                    x.x = u00r * a.x - u00i * a.y + u01r * b.x - u01i * b.y;
                    x.y = u00r * a.y + u00i * a.x + u01r * b.y + u01i * b.x;
                    y.x = u10r * a.x - u10i * a.y + u11r * b.x - u11i * b.y;
                    y.y = u10r * a.y + u10i * a.x + u11r * b.y + u11i * b.x;
                    buf[e0] = x;
                    buf[e1] = y;
                }
            }
            __syncthreads();
        }

        // ---- write back ----
        if (direct) {
            for (uint32_t e = uint32_t(tid); e < tile_elems; e += kThreads)
                state[chunk_base(g, r, e >> g.c) + (e & ((1u << g.c) - 1u))] = buf[e];
            __syncthreads();
            continue;
        }
        fence_proxy_async();
        __syncthreads();
        if (warp == 0) issue_tile_store(g, state, buf, r, lane);
    }
    if (!direct && warp == 0) bulk_wait0();
}

// ---------------------------------------------------------------------------
// get_state scatter

template <typename E>
__global__ void __launch_bounds__(kThreads) scatter_kernel(const E *__restrict__ state, uint64_t n_real,
                                                           const uint64_t *__restrict__ coltab, uint64_t b, int N,
                                                           int order, double gre, double gim, E *__restrict__ out)
{
    using R = typename ET<E>::R;
    __shared__ uint64_t tab[8][256];
    for (int i = threadIdx.x; i < 8 * 256; i += kThreads) tab[i >> 8][i & 255] = coltab[i];
    __syncthreads();
    const R gr = R(gre), gi = R(gim);
    for (uint64_t r = uint64_t(blockIdx.x) * kThreads + threadIdx.x; r < n_real; r += uint64_t(gridDim.x) * kThreads) {
        uint64_t v = b;
#pragma unroll
        for (int k = 0; k < 8; k++) v ^= tab[k][(r >> (8 * k)) & 255];
        const uint64_t idx = order == 0 ? (__brevll(v) >> (64 - N)) : v;
        const E a = state[r];
        E o;
        o.x = a.x * gr - a.y * gi;
        o.y = a.x * gi + a.y * gr;
        out[idx] = o;
    }
}

// ---------------------------------------------------------------------------
// launchers

template <typename E>
static cudaError_t launch_tile(const uint8_t *blob, uint64_t off, uint32_t T, uint64_t ntiles, E *state,
                               DevStatus *status, int sms, cudaStream_t st)
{
    const size_t smem = 2 * (sizeof(E) << T);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(tile_kernel<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
    }
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tile_kernel<E>, kThreads, smem);
    if (per_sm < 1) per_sm = 1;
    uint64_t grid = uint64_t(sms) * uint64_t(per_sm);
    if (grid > ntiles) grid = ntiles;
    tile_kernel<E><<<unsigned(grid), kThreads, smem, st>>>(blob, off, state, status);
    return cudaGetLastError();
}

namespace {
template <typename E>
__global__ void set_one_kernel(E *state)
{
    state[0].x = 1;
    state[0].y = 0;
}
}  // namespace

cudaError_t run_set_one(void *state, int elem_bytes, cudaStream_t st)
{
    if (elem_bytes == 8) set_one_kernel<float2><<<1, 1, 0, st>>>(static_cast<float2 *>(state));
    else set_one_kernel<double2><<<1, 1, 0, st>>>(static_cast<double2 *>(state));
    return cudaGetLastError();
}

cudaError_t run_passes(const std::vector<Pass> &passes, const uint8_t *dblob, void *state, int elem_bytes,
                       DevStatus *status, int sms, cudaStream_t st, uint64_t &kernels, const void *first_src,
                       void *last_dst)
{
    for (size_t i = 0; i < passes.size(); i++) {
        const Pass &ps = passes[i];
        cudaError_t e = cudaSuccess;
        if (ps.kind == Pass::PRODUCT) {
            const uint64_t nvec = std::max<uint64_t>(1, (1ULL << ps.m) / (16 / elem_bytes));
            const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((nvec + kThreads - 1) / kThreads,
                                                                                    uint64_t(sms) * 8)));
            if (elem_bytes == 8)
                product_kernel<float2><<<grid, kThreads, 0, st>>>(dblob, ps.off, ps.off2, static_cast<float2 *>(state));
            else
                product_kernel<double2><<<grid, kThreads, 0, st>>>(dblob, ps.off, ps.off2, static_cast<double2 *>(state));
            e = cudaGetLastError();
        } else if (ps.kind == Pass::EXPAND) {
            const uint64_t half = 1ULL << (ps.m - 1);
            const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((half + kThreads - 1) / kThreads,
                                                                                    uint64_t(sms) * 16)));
            if (elem_bytes == 8)
                expand_kernel<float2><<<grid, kThreads, 0, st>>>(dblob, ps.off, static_cast<float2 *>(state));
            else
                expand_kernel<double2><<<grid, kThreads, 0, st>>>(dblob, ps.off, static_cast<double2 *>(state));
            e = cudaGetLastError();
        } else if (ps.kind == Pass::ROW) {
            e = run_row_pass(dblob, ps.off, ps.off2, ps.row.nitems, elem_bytes, ps.wide, ps.low != 0, ps.real != 0,
                             ps.row.off_pre != 0 || ps.row.off_post != 0, state, sms, st);
        } else if (ps.kind == Pass::FAST) {
            e = run_fast_tile(dblob, ps.off, ps.off2, ps.geom.ntiles, elem_bytes, state, status, sms, st);
        } else if (ps.kind == Pass::INIT) {
            const size_t bytes = size_t(elem_bytes) << ps.m;
            e = cudaMemsetAsync(state, 0, bytes, st);
            if (e == cudaSuccess) e = run_set_one(state, elem_bytes, st);
        } else if (ps.kind == Pass::GROW) {
            // out of place at the ends when asked: read the first pass from first_src,
            // write the last pass to last_dst (reading state)
            void *dst = (i + 1 == passes.size() && last_dst) ? last_dst : state;
            const void *src = (i == 0 && first_src) ? first_src : (dst != state ? state : nullptr);
            e = run_grow(dblob, ps.off, ps.off2, int(ps.gb.regs.size()), ps.gb.dev.nitems, elem_bytes, dst, nullptr,
                         nullptr, ps.gb.all_real(), ps.prefetch != 0, status, sms, st, src);
        } else if (ps.kind == Pass::DIAG) {
            e = run_diag(dblob, ps.off, ps.off2, ps.m, elem_bytes, ps.row_bits, ps.chunk_bits, ps.prefetch != 0, state, status,
                         sms, st);
        } else if (ps.kind == Pass::SPAN) {
            e = run_span(dblob, ps.off, ps.off2, ps.span.ntiles, elem_bytes, ps.low != 0,
                         span_layouts(elem_bytes, ps.span.gates, ps.low != 0, ps.prefetch != 0), ps.prefetch != 0,
                         ps.real, state, ps.span.rot, ps.span.pos, sms, st);
        } else if (ps.kind == Pass::WALSH) {
            e = run_walsh(dblob, ps.off, ps.off2, ps.m, uint32_t(ps.row_bits), elem_bytes, state, sms, st);
        } else if (ps.kind == Pass::PAIR) {
            const uint64_t np = 1ULL << (ps.m - 1);
            const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((np + kThreads - 1) / kThreads,
                                                                                    uint64_t(sms) * 16)));
            if (elem_bytes == 8)
                pair_kernel<float2><<<grid, kThreads, 0, st>>>(dblob, ps.off, static_cast<float2 *>(state));
            else
                pair_kernel<double2><<<grid, kThreads, 0, st>>>(dblob, ps.off, static_cast<double2 *>(state));
            e = cudaGetLastError();
        } else {
            if (elem_bytes == 8)
                e = launch_tile<float2>(dblob, ps.off, ps.geom.T, ps.geom.ntiles, static_cast<float2 *>(state), status,
                                        sms, st);
            else
                e = launch_tile<double2>(dblob, ps.off, ps.geom.T, ps.geom.ntiles, static_cast<double2 *>(state), status,
                                         sms, st);
        }
        if (e != cudaSuccess) return e;
        kernels++;
    }
    return cudaSuccess;
}

cudaError_t run_scatter(const void *state, uint64_t n_real, const uint64_t *dcoltab, uint64_t b, int N, int order,
                        double gre, double gim, void *out, int elem_bytes, int sms, cudaStream_t st)
{
    const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((n_real + kThreads - 1) / kThreads,
                                                                            uint64_t(sms) * 16)));
    if (elem_bytes == 8)
        scatter_kernel<float2><<<grid, kThreads, 0, st>>>(static_cast<const float2 *>(state), n_real, dcoltab, b, N,
                                                          order, gre, gim, static_cast<float2 *>(out));
    else
        scatter_kernel<double2><<<grid, kThreads, 0, st>>>(static_cast<const double2 *>(state), n_real, dcoltab, b, N,
                                                           order, gre, gim, static_cast<double2 *>(out));
    return cudaGetLastError();
}

}  // namespace zxh
