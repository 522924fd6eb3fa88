// lambda_dev.cuh -- lambda = H psi and <psi|H|psi> for a sum of Z, ZZ and X terms
// on the real-address state, shared by the adjoint sweep's lambda_kernel
// (adjoint.cu) and the persistent batch kernel's lambda op (batch.cu).
//
// A virtual Z_q is the selector S_q(r) = parity(alpha_q & r) ^ beta_q of the
// affine map, so a Z or ZZ term is +-c by the parity of r & m (m the xor of its
// selectors' masks, the sign from their offsets) and needs no memory access; a
// virtual X_q flips the real address by delta_q (A delta_q = e_q) and gathers
// psi[r ^ delta_q]. The reference evaluates the observable on the host after
// get_state; this runs on the device in one pass over the state.
//
// Layout of the work: a warp takes 256 consecutive amplitudes, 8 per lane (lane,
// lane + 32, ...), so every term is read from shared memory once per 8
// amplitudes, every gather is a coalesced 256-byte warp access, and a term's
// parity splits into the 256-block's part (one 64-bit parity per term) and the
// low 8 bits' part (one 32-bit popcount per amplitude).
#pragma once

#include "adjoint.h"
#include "core.h"
#include "dev.cuh"

#include <cuda_runtime.h>

namespace zxh {
namespace ldev {

template <typename E>
struct LamTables {
    using R = typename ET<E>::R;
    uint64_t xd[kMaxTerms];  // X terms: the real-address flip
    R xc[kMaxTerms];
    uint64_t dm[kMaxTerms];  // Z / ZZ terms: the selector mask (ZZ: both masks xored)
    R dc[kMaxTerms];         // the coefficient, negated where the selector offsets xor to 1
    uint32_t nx, nd;
};

// All threads of the CTA; the host lists X terms first. Ends with a barrier.
template <typename E>
__device__ __forceinline__ void lam_load(LamTables<E> &t, const TermDev *terms, uint32_t nterms)
{
    using R = typename ET<E>::R;
    if (threadIdx.x == 0) {
        uint32_t k = 0;
        while (k < nterms && terms[k].kind == 3) k++;
        t.nx = k;
        t.nd = nterms - k;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nterms; i += blockDim.x) {
        const TermDev tm = terms[i];
        if (i < t.nx) {
            t.xd[i] = tm.delta;
            t.xc[i] = R(tm.coef);
        } else {
            uint64_t m = tm.a0;
            uint32_t b = tm.b0;
            if (tm.kind == 2) {
                m ^= tm.a1;
                b ^= tm.b1;
            }
            t.dm[i - t.nx] = m;
            t.dc[i - t.nx] = (b & 1) ? -R(tm.coef) : R(tm.coef);
        }
    }
    __syncthreads();
}

template <bool CG, typename E>
__device__ __forceinline__ E lam_ld(const E *p)
{
    if constexpr (CG) return __ldcg(p);
    else return __ldg(p);
}

// lambda on the amplitudes [b, e) of the 256-blocks gw, gw + nw, ... (counted
// from the block holding b); returns this thread's share of Re <psi|lambda> in
// FP64. lambda is accumulated in the state's precision (it is stored in it).
// CG: loads and stores through L2 only (the batch kernel, whose other SMs wrote
// psi in the previous op).
template <typename E, bool WRITE, bool CG>
__device__ __forceinline__ double lam_rows(const E *__restrict__ psi, E *__restrict__ lam, uint64_t b, uint64_t e,
                                           const LamTables<E> &t, uint64_t gw, uint64_t nw)
{
    using R = typename ET<E>::R;
    constexpr int A = 8;
    const uint32_t lane = threadIdx.x & 31u;
    double en = 0.0;
    for (uint64_t blk = (b >> 8) + gw; (blk << 8) < e; blk += nw) {
        const uint64_t base = blk << 8;
        E p[A];
        R dg[A], xr[A], xi[A];
        bool ok[A];
#pragma unroll
        for (int j = 0; j < A; j++) {
            const uint64_t r = base + uint64_t(32 * j) + lane;
            ok[j] = r >= b && r < e;
            p[j] = ok[j] ? lam_ld<CG>(psi + r) : E{0, 0};
            dg[j] = 0;
            xr[j] = 0;
            xi[j] = 0;
        }
        for (uint32_t k = 0; k < t.nx; k++) {
            const uint64_t d = t.xd[k];
            const R c = t.xc[k];
#pragma unroll
            for (int j = 0; j < A; j++)
                if (ok[j]) {
                    const E q = lam_ld<CG>(psi + ((base + uint64_t(32 * j) + lane) ^ d));
                    xr[j] += c * q.x;
                    xi[j] += c * q.y;
                }
        }
        for (uint32_t k = 0; k < t.nd; k++) {
            const uint64_t m = t.dm[k];
            const R c = t.dc[k];
            const uint32_t hp = uint32_t(par64(base & m));
            const uint32_t ml = uint32_t(m) & 255u;
#pragma unroll
            for (int j = 0; j < A; j++) {
                const uint32_t s = hp ^ (uint32_t(__popc((uint32_t(32 * j) + lane) & ml)) & 1u);
                dg[j] += s ? -c : c;
            }
        }
#pragma unroll
        for (int j = 0; j < A; j++) {
            if (!ok[j]) continue;
            E l;
            l.x = dg[j] * p[j].x + xr[j];
            l.y = dg[j] * p[j].y + xi[j];
            if constexpr (WRITE) {
                if constexpr (CG) __stcg(lam + base + uint64_t(32 * j) + lane, l);
                else lam[base + uint64_t(32 * j) + lane] = l;
            }
            en += double(p[j].x) * double(l.x) + double(p[j].y) * double(l.y);  // Re(conj(psi) lambda)
        }
    }
    return en;
}

}  // namespace ldev
}  // namespace zxh
