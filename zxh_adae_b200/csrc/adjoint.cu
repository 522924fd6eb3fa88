// adjoint.cu -- expectation values and the adjoint-gradient reverse sweep (sm_100a).
//
// No counterpart in the reference (ZXH-Sim has no observables). Everything works
// on the real-address state: a virtual Z_q is the selector S_q(r) of the affine
// map, a virtual X_q flips the real address by delta_q (A delta_q = e_q).
//
//   lambda_kernel     lambda = H psi for a sum of Z, ZZ and X terms, and <psi|H|psi>
//                     reduced in FP64 in the same pass (lambda_dev.cuh).
//   adj_pair_kernel   one rotation (or any 2x2 gate) of the reverse sweep: its
//                     gradient Im<lambda|G|psi> reduced in FP64, then psi and
//                     lambda uncomputed with U^dagger, one read-modify-write of both.
//   adj_diag_kernel   a group of commuting diagonal gates (RZ, P, CP, Z): all their
//                     gradients reduced in one pass, then both states multiplied
//                     by the inverse phase.
#include "adjoint.h"
#include "core.h"
#include "dev.cuh"
#include "lambda_dev.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

namespace zxh {

namespace {

template <typename E>
__device__ __forceinline__ double dre(const E &a) { return double(a.x); }
template <typename E>
__device__ __forceinline__ double dim(const E &a) { return double(a.y); }

__device__ __forceinline__ double block_sum(double v, double *sh)
{
    v = warp_sum_f64(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kThreads / 32; w++) t += sh[w];
    __syncthreads();
    return t;
}

template <typename E, bool WRITE>
__global__ void __launch_bounds__(kThreads) lambda_kernel(const E *__restrict__ psi, E *__restrict__ lam, uint64_t n,
                                                          const TermDev *__restrict__ terms, uint32_t nterms,
                                                          double *energy)
{
    __shared__ ldev::LamTables<E> t;
    __shared__ double sh[kThreads / 32];
    ldev::lam_load(t, terms, nterms);
    const uint64_t gw = uint64_t(blockIdx.x) * (kThreads / 32) + (threadIdx.x >> 5);
    const uint64_t nw = uint64_t(gridDim.x) * (kThreads / 32);
    double en = ldev::lam_rows<E, WRITE, false>(psi, lam, 0, n, t, gw, nw);
    en = block_sum(en, sh);
    if (threadIdx.x == 0) atomicAdd(energy, en);
}

template <typename E>
__global__ void __launch_bounds__(kThreads) adj_pair_kernel(E *__restrict__ psi, E *__restrict__ lam, AdjPairDev g,
                                                            double *grad)
{
    using R = typename ET<E>::R;
    __shared__ double sh[kThreads / 32];
    const uint64_t npairs = 1ULL << (g.m - 1);
    const uint32_t pv = g.pivot;
    // U^dagger = [[conj u00, conj u10], [conj u01, conj u11]]
    const R a00r = R(g.u[0]), a00i = R(-g.u[1]), a01r = R(g.u[4]), a01i = R(-g.u[5]);
    const R a10r = R(g.u[2]), a10i = R(-g.u[3]), a11r = R(g.u[6]), a11i = R(-g.u[7]);
    double gacc = 0.0;
    for (uint64_t q = uint64_t(blockIdx.x) * kThreads + threadIdx.x; q < npairs; q += uint64_t(gridDim.x) * kThreads) {
        uint64_t e0 = ((q >> pv) << (pv + 1)) | (q & ((1ULL << pv) - 1ULL));
        uint64_t e1 = e0 ^ g.delta;
        if (par64(g.alpha & e0) ^ int(g.beta)) {
            const uint64_t t = e0;
            e0 = e1;
            e1 = t;
        }
        const E pe = psi[e0], po = psi[e1], le = lam[e0], lo = lam[e1];
        if (g.gen == 1) {  // Im<lambda|Y|psi> = Re(conj(lo) pe) - Re(conj(le) po)
            gacc += dre(lo) * dre(pe) + dim(lo) * dim(pe) - dre(le) * dre(po) - dim(le) * dim(po);
        } else if (g.gen == 2) {  // Im<lambda|X|psi> = Im(conj(le) po + conj(lo) pe)
            gacc += dre(le) * dim(po) - dim(le) * dre(po) + dre(lo) * dim(pe) - dim(lo) * dre(pe);
        }
        E x, y;
        x.x = a00r * pe.x - a00i * pe.y + a01r * po.x - a01i * po.y;
        x.y = a00r * pe.y + a00i * pe.x + a01r * po.y + a01i * po.x;
        y.x = a10r * pe.x - a10i * pe.y + a11r * po.x - a11i * po.y;
        y.y = a10r * pe.y + a10i * pe.x + a11r * po.y + a11i * po.x;
        psi[e0] = x;
        psi[e1] = y;
        x.x = a00r * le.x - a00i * le.y + a01r * lo.x - a01i * lo.y;
        x.y = a00r * le.y + a00i * le.x + a01r * lo.y + a01i * lo.x;
        y.x = a10r * le.x - a10i * le.y + a11r * lo.x - a11i * lo.y;
        y.y = a10r * le.y + a10i * le.x + a11r * lo.y + a11i * lo.x;
        lam[e0] = x;
        lam[e1] = y;
    }
    if (g.gen) {
        gacc = block_sum(gacc, sh);
        if (threadIdx.x == 0) atomicAdd(grad, gacc);
    }
}

template <int NG>
struct AdjDiagParams {
    AdjDiagGate g[NG];
    uint32_t slot[NG];
    uint32_t ng;
};

// The group's gates travel as a kernel parameter, so every gate field is a
// constant-bank operand of the instructions that use it rather than a register.
template <typename E, int NG>
__global__ void __launch_bounds__(kThreads) adj_diag_kernel(E *__restrict__ psi, E *__restrict__ lam, uint64_t n,
                                                            const __grid_constant__ AdjDiagParams<NG> P,
                                                            double *grads, const E *__restrict__ exp_tab)
{
    __shared__ E s_exp[1 << kExpTableBits];
    __shared__ double sh[kThreads / 32];
    for (int i = threadIdx.x; i < (1 << kExpTableBits); i += kThreads) s_exp[i] = exp_tab[i];
    __syncthreads();
    double acc[NG];
#pragma unroll
    for (int j = 0; j < NG; j++) acc[j] = 0.0;
    for (uint64_t r = uint64_t(blockIdx.x) * kThreads + threadIdx.x; r < n; r += uint64_t(gridDim.x) * kThreads) {
        const E p = psi[r], l = lam[r];
        const double w = dre(l) * dim(p) - dim(l) * dre(p);  // Im(conj(lambda) psi)
        int64_t th = 0;
#pragma unroll
        for (int j = 0; j < NG; j++) {
            if (j >= int(P.ng)) break;
            const AdjDiagGate &G = P.g[j];
            const int s0 = par64(r & G.a0) ^ int(G.b0);
            const int s = G.two ? (s0 & (par64(r & G.a1) ^ int(G.b1))) : s0;
            acc[j] = fma(w, s ? G.m1 : G.m0, acc[j]);
            th += s ? G.tq : 0;
        }
        E ph;
        if constexpr (ET<E>::V == 2) ph = phase_factor32(s_exp, turns32(-th));
        else ph = phase_factor(s_exp, -th);
        psi[r] = cmul(p, ph);
        lam[r] = cmul(l, ph);
    }
#pragma unroll
    for (int j = 0; j < NG; j++) {
        if (j >= int(P.ng)) break;
        const double t = block_sum(acc[j], sh);
        if (threadIdx.x == 0 && P.g[j].kind) atomicAdd(&grads[P.slot[j]], t);
    }
}

unsigned grid_for(uint64_t work, int sms)
{
    return unsigned(std::max<uint64_t>(1, std::min<uint64_t>((work + kThreads - 1) / kThreads, uint64_t(sms) * 8)));
}

}  // namespace

cudaError_t run_lambda(const void *psi, void *lam, int m, int elem_bytes, const TermDev *dterms, uint32_t nterms,
                       double *energy, int sms, cudaStream_t st)
{
    const uint64_t n = 1ULL << m;
    // a warp takes 256 amplitudes at a time (8 per lane)
    const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((n + 2047) / 2048, uint64_t(sms) * 8)));
    if (elem_bytes == 8) {
        auto p = static_cast<const float2 *>(psi);
        auto l = static_cast<float2 *>(lam);
        if (lam) lambda_kernel<float2, true><<<grid, kThreads, 0, st>>>(p, l, n, dterms, nterms, energy);
        else lambda_kernel<float2, false><<<grid, kThreads, 0, st>>>(p, l, n, dterms, nterms, energy);
    } else {
        auto p = static_cast<const double2 *>(psi);
        auto l = static_cast<double2 *>(lam);
        if (lam) lambda_kernel<double2, true><<<grid, kThreads, 0, st>>>(p, l, n, dterms, nterms, energy);
        else lambda_kernel<double2, false><<<grid, kThreads, 0, st>>>(p, l, n, dterms, nterms, energy);
    }
    return cudaGetLastError();
}

cudaError_t run_adj_pair(void *psi, void *lam, int elem_bytes, const AdjPairDev &g, double *grad, int sms,
                         cudaStream_t st)
{
    const uint64_t np = 1ULL << (g.m - 1);
    if (elem_bytes == 8)
        adj_pair_kernel<float2><<<grid_for(np, sms), kThreads, 0, st>>>(static_cast<float2 *>(psi),
                                                                       static_cast<float2 *>(lam), g, grad);
    else
        adj_pair_kernel<double2><<<grid_for(np, sms), kThreads, 0, st>>>(static_cast<double2 *>(psi),
                                                                        static_cast<double2 *>(lam), g, grad);
    return cudaGetLastError();
}

namespace {

template <typename E, int NG>
cudaError_t launch_adj_diag(E *psi, E *lam, uint64_t n, const AdjDiagGate *gates, uint32_t ng, double *grads,
                            const uint32_t *slots, const void *exp_tab, int sms, cudaStream_t st)
{
    AdjDiagParams<NG> P;
    std::memset(&P, 0, sizeof(P));
    for (uint32_t j = 0; j < ng; j++) {
        P.g[j] = gates[j];
        P.slot[j] = slots[j];
    }
    P.ng = ng;
    adj_diag_kernel<E, NG><<<grid_for(n, sms), kThreads, 0, st>>>(psi, lam, n, P, grads, static_cast<const E *>(exp_tab));
    return cudaGetLastError();
}

template <typename E>
cudaError_t adj_diag_typed(E *psi, E *lam, uint64_t n, const AdjDiagGate *gates, uint32_t ng, double *grads,
                           const uint32_t *slots, const void *exp_tab, int sms, cudaStream_t st)
{
    if (ng <= 8) return launch_adj_diag<E, 8>(psi, lam, n, gates, ng, grads, slots, exp_tab, sms, st);
    if (ng <= 16) return launch_adj_diag<E, 16>(psi, lam, n, gates, ng, grads, slots, exp_tab, sms, st);
    if (ng <= uint32_t(kAdjDiagMax))
        return launch_adj_diag<E, kAdjDiagMax>(psi, lam, n, gates, ng, grads, slots, exp_tab, sms, st);
    return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t run_adj_diag(void *psi, void *lam, int m, int elem_bytes, const AdjDiagGate *gates, uint32_t ng,
                         double *grads, const uint32_t *slots, const void *exp_tab, int sms, cudaStream_t st)
{
    const uint64_t n = 1ULL << m;
    if (elem_bytes == 8)
        return adj_diag_typed(static_cast<float2 *>(psi), static_cast<float2 *>(lam), n, gates, ng, grads, slots,
                              exp_tab, sms, st);
    return adj_diag_typed(static_cast<double2 *>(psi), static_cast<double2 *>(lam), n, gates, ng, grads, slots,
                          exp_tab, sms, st);
}

}  // namespace zxh
