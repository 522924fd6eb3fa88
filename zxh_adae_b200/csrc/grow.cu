// grow.cu -- the general strided pass (sm_100a): a batch of single-qubit gates
// whose pair deltas span several real bits (the state after CX transport through
// the affine map), with diagonal windows fused before and after.
//
// The reference applies every such gate as its own grid sweep over the state with
// a cooperative grid.sync() between them (u3_block_batch_kernel_cuda,
// src/zxh/src/kernel/kernel_cuda.cu:390-423). Here one pass applies up to R gates
// with multi-bit deltas (R register coordinates) plus any number of gates whose
// delta lies in the low F bits (lane gates), with one read and one write of every
// amplitude:
//
// * Row k of a thread holds the amplitudes at r0 ^ D[k] ^ (lane, vector slot),
//   D[k] = xor of the deltas delta_i over the set bits i of k. The partner of an
//   amplitude under gate i is then the same lane and slot in row k ^ e_i, so the
//   2x2 update is register-local. A warp's loads of one row are a permutation of
//   512 contiguous bytes (coalesced).
// * The selector of any qubit's row is parity(alpha & r0) ^ (lane part) ^ (row
//   part); the first is one parity per lane and item (ballot), the second a
//   per-thread constant, the third is nonzero only for the pass's own register
//   qubits. Gate orientation and window phases follow from these bits; a
//   window's phase over a thread's rows is a polynomial in the row bits (constant,
//   linear, pairwise), summed per row at compile-time positions.
// * Adjoint mode (two states psi, lambda): each gate's gradient Im<lambda|G|psi>
//   is reduced in FP64 right before its U^dagger is applied to both states; the
//   pass's gates act on distinct qubits and commute, so that is the gradient at
//   the group's end, as the adjoint method needs.
#include "core.h"
#include "dev.cuh"
#include "grow_dev.cuh"
#include "host.h"
#include "sampler.h"

#include <algorithm>
#include <cuda_runtime.h>

namespace zxh {

namespace {

using namespace gdev;

// The adjoint pass with 4 register coordinates holds 16 rows of both states: one
// CTA per SM (twice the rows in flight per warp, the same bytes per SM). PF: the
// staged form (next item's rows copied into shared memory during the current one).
template <typename E, int R, bool ADJ, bool REAL, bool PF>
__global__ void __launch_bounds__(kThreads, (ADJ && R == 4) ? 1 : 2)
    grow_kernel(const uint8_t *__restrict__ blob, uint64_t poff, uint64_t toff, E *__restrict__ psi,
                E *__restrict__ lam, double *grads, uint64_t nitems, DevStatus *status, const E *psi_src)
{
    __shared__ GrowShared<E> sm;
    extern __shared__ __align__(128) uint8_t stage[];
    constexpr int WARPS = kThreads / 32;
    grow_body<E, R, ADJ, REAL, PF>(blob, poff, toff, psi, lam, grads, uint64_t(blockIdx.x) * WARPS,
                                   uint64_t(gridDim.x) * WARPS, nitems, sm, stage, status, psi_src);
}

template <typename E, int R, bool ADJ, bool REAL, bool PF>
cudaError_t launch_grow(const uint8_t *dblob, uint64_t poff, uint64_t toff, uint64_t nitems, E *psi, E *lam,
                        double *grads, DevStatus *status, const E *psi_src, int sms, cudaStream_t st)
{
    auto kern = grow_kernel<E, R, ADJ, REAL, PF>;
    const size_t smem = PF ? grow_stage_bytes<R, ADJ>() : 0;
    if (PF) {
        const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
    }
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
    if (per_sm < 1) per_sm = 1;
    const uint64_t ctas = (nitems + kThreads / 32 - 1) / (kThreads / 32);
    const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(ctas, uint64_t(sms) * uint64_t(per_sm))));
    kern<<<grid, kThreads, smem, st>>>(dblob, poff, toff, psi, lam, grads, nitems, status, psi_src);
    return cudaGetLastError();
}

template <typename E, bool ADJ, bool REAL, bool PF>
cudaError_t grow_typed(int R, const uint8_t *dblob, uint64_t poff, uint64_t toff, uint64_t nitems, E *psi, E *lam,
                       double *grads, DevStatus *status, const E *psi_src, int sms, cudaStream_t st)
{
    switch (R) {
    case 0: return launch_grow<E, 0, ADJ, REAL, PF>(dblob, poff, toff, nitems, psi, lam, grads, status, psi_src, sms, st);
    case 1: return launch_grow<E, 1, ADJ, REAL, PF>(dblob, poff, toff, nitems, psi, lam, grads, status, psi_src, sms, st);
    case 2: return launch_grow<E, 2, ADJ, REAL, PF>(dblob, poff, toff, nitems, psi, lam, grads, status, psi_src, sms, st);
    case 3: return launch_grow<E, 3, ADJ, REAL, PF>(dblob, poff, toff, nitems, psi, lam, grads, status, psi_src, sms, st);
    case 4: return launch_grow<E, 4, ADJ, REAL, PF>(dblob, poff, toff, nitems, psi, lam, grads, status, psi_src, sms, st);
    default: return cudaErrorInvalidValue;
    }
}

template <typename E, bool ADJ>
cudaError_t grow_real(bool real, bool staged, int R, const uint8_t *dblob, uint64_t poff, uint64_t toff,
                      uint64_t nitems, E *psi, E *lam, double *grads, DevStatus *status, const E *src, int sms,
                      cudaStream_t st)
{
    if (staged)
        return real ? grow_typed<E, ADJ, true, true>(R, dblob, poff, toff, nitems, psi, lam, grads, status, src, sms, st)
                    : grow_typed<E, ADJ, false, true>(R, dblob, poff, toff, nitems, psi, lam, grads, status, src, sms, st);
    return real ? grow_typed<E, ADJ, true, false>(R, dblob, poff, toff, nitems, psi, lam, grads, status, src, sms, st)
                : grow_typed<E, ADJ, false, false>(R, dblob, poff, toff, nitems, psi, lam, grads, status, src, sms, st);
}

}  // namespace

int grow_reg_bits(int elem_bytes, bool adjoint)
{
    (void)elem_bytes;
    return adjoint ? 4 : 4;  // the most the kernels take; the adjoint sweep picks 3 or 4 (adj_regs)
}

int grow_fixed_bits(int elem_bytes) { return elem_bytes == 8 ? 6 : 5; }

int grow_adjoint_gates() { return kGrowAdjGates; }

cudaError_t run_grow(const uint8_t *dblob, uint64_t poff, uint64_t toff, int R, uint64_t nitems, int elem_bytes,
                     void *psi, void *lam, double *grads, bool real, bool staged, DevStatus *status, int sms,
                     cudaStream_t st, const void *psi_src)
{
    const bool adj = lam != nullptr;
    staged = staged && status != nullptr;
    if (elem_bytes == 8) {
        auto *a = static_cast<float2 *>(psi);
        auto *b = static_cast<float2 *>(lam);
        auto *c = static_cast<const float2 *>(psi_src);
        return adj ? grow_real<float2, true>(real, staged, R, dblob, poff, toff, nitems, a, b, grads, status, c, sms, st)
                   : grow_real<float2, false>(real, staged, R, dblob, poff, toff, nitems, a, b, grads, status, c, sms, st);
    }
    auto *a = static_cast<double2 *>(psi);
    auto *b = static_cast<double2 *>(lam);
    auto *c = static_cast<const double2 *>(psi_src);
    return adj ? grow_real<double2, true>(real, staged, R, dblob, poff, toff, nitems, a, b, grads, status, c, sms, st)
               : grow_real<double2, false>(real, staged, R, dblob, poff, toff, nitems, a, b, grads, status, c, sms, st);
}

}  // namespace zxh
