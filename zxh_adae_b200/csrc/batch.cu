// batch.cu -- the persistent batch kernel (sm_100a) and the per-op launches of
// the sequential comparison.
//
// No counterpart in the reference (one circuit per ZXH object, process-global
// state, kernel_cuda.cu:91-142). Each CTA loops: take the next task from the
// queue head (one atomic), wait until the op it depends on (the previous pass of
// the same circuit) has no task left (bounded spin on a counter; a timeout sets
// the status word and ends the kernel), run the task's slice of the op, and
// count the task done. The queue lists every op's tasks after those of the op it
// depends on, so the tasks a CTA waits for were taken earlier by CTAs that are
// running: no co-residency is needed. State loads and stores go through L2
// (.cg), and each task fences its stores before it is counted.
#include "batch.h"
#include "dev.cuh"
#include "grow_dev.cuh"
#include "lambda_dev.cuh"

#include <algorithm>
#include <cuda_runtime.h>

namespace zxh {

namespace {

using namespace gdev;

// NT: threads of the persistent kernel's CTA (the warps that work on one task).
template <typename E, int NT>
struct LamShared {
    ldev::LamTables<E> t;
    double red[NT / 32];
};

template <typename E, int NT>
struct DiagShared {
    AdjDiagGate g[kBatchDiagMax];
    uint32_t slot[kBatchDiagMax];
    E exp[1 << kExpTableBits];
    double red[NT / 32];
};

template <typename E, int NT>
union BatchShared {
    GrowShared<E, NT> g;
    LamShared<E, NT> l;
    DiagShared<E, NT> d;
};

template <typename E>
__device__ __forceinline__ double re_d(E a) { return double(a.x); }
template <typename E>
__device__ __forceinline__ double im_d(E a) { return double(a.y); }

template <int NT>
__device__ __forceinline__ double cta_sum(double v, double *red)
{
    v = warp_sum_f64(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < NT / 32; w++) t += red[w];
    return t;
}

template <typename E, int NT>
__device__ __forceinline__ void init_body(E *psi, uint64_t b, uint64_t e)
{
    for (uint64_t i = b + threadIdx.x; i < e; i += NT) {
        E v;
        v.x = i == 0 ? 1 : 0;
        v.y = 0;
        __stcg(psi + i, v);
    }
}

template <typename E, int NT>
__device__ __forceinline__ void lambda_body(const E *psi, E *lam, uint64_t b, uint64_t e, const TermDev *terms,
                                            uint32_t nterms, double *energy, LamShared<E, NT> &sm)
{
    __syncthreads();  // the shared tables may still be read by a previous op
    ldev::lam_load(sm.t, terms, nterms);
    double en = ldev::lam_rows<E, true, true>(psi, lam, b, e, sm.t, threadIdx.x >> 5, NT / 32);
    en = cta_sum<NT>(en, sm.red);
    if (threadIdx.x == 0) atomicAdd(energy, en);
}

template <typename E, int NT>
__device__ __forceinline__ void diag_adj_body(E *psi, E *lam, uint64_t b, uint64_t e, const AdjDiagGate *gates,
                                              const uint32_t *slots, uint32_t ng, const E *exp_tab, double *grads,
                                              DiagShared<E, NT> &sm)
{
    __syncthreads();
    if (threadIdx.x < ng) {
        sm.g[threadIdx.x] = gates[threadIdx.x];
        sm.slot[threadIdx.x] = slots[threadIdx.x];
    }
    for (int i = threadIdx.x; i < (1 << kExpTableBits); i += NT) sm.exp[i] = exp_tab[i];
    __syncthreads();
    double acc[kBatchDiagMax];
#pragma unroll
    for (int j = 0; j < kBatchDiagMax; j++) acc[j] = 0.0;
    for (uint64_t r = b + threadIdx.x; r < e; r += NT) {
        const E p = __ldcg(psi + r), l = __ldcg(lam + r);
        const double w = re_d(l) * im_d(p) - im_d(l) * re_d(p);  // Im(conj(lambda) psi)
        int64_t th = 0;
#pragma unroll
        for (int j = 0; j < kBatchDiagMax; j++) {
            if (j >= int(ng)) break;
            const AdjDiagGate &G = sm.g[j];
            const int s0 = par64(r & G.a0) ^ int(G.b0);
            const int s = G.two ? (s0 & (par64(r & G.a1) ^ int(G.b1))) : s0;
            acc[j] = fma(w, s ? G.m1 : G.m0, acc[j]);
            th += s ? G.tq : 0;
        }
        E ph;
        if constexpr (ET<E>::V == 2) ph = phase_factor32(sm.exp, turns32(-th));
        else ph = phase_factor(sm.exp, -th);
        __stcg(psi + r, cmul(p, ph));
        __stcg(lam + r, cmul(l, ph));
    }
#pragma unroll
    for (int j = 0; j < kBatchDiagMax; j++) {
        if (j >= int(ng)) break;
        const double t = cta_sum<NT>(acc[j], sm.red);
        if (threadIdx.x == 0 && sm.g[j].kind) atomicAdd(&grads[sm.slot[j]], t);
    }
}

template <typename E, bool REAL, int NT>
__device__ __forceinline__ void run_op_slice(const BatchOp &op, const uint8_t *blob, E *arena, double *grads,
                                             double *energies, uint64_t b, uint64_t e, uint64_t first, uint64_t step,
                                             BatchShared<E, NT> &sm)
{
    const uint8_t *ob = blob + op.base;
    E *psi = arena + op.psi;
    E *lam = arena + op.lam;
    double *gr = grads + op.grad_base;
    switch (op.kind) {
    case BOP_INIT: init_body<E, NT>(psi, b, e); break;
    case BOP_GROW:
        switch (op.R) {
        case 0: grow_body<E, 0, false, REAL, false, NT>(ob, op.off0, op.off1, psi, nullptr, nullptr, first, step, e, sm.g); break;
        case 1: grow_body<E, 1, false, REAL, false, NT>(ob, op.off0, op.off1, psi, nullptr, nullptr, first, step, e, sm.g); break;
        case 2: grow_body<E, 2, false, REAL, false, NT>(ob, op.off0, op.off1, psi, nullptr, nullptr, first, step, e, sm.g); break;
        case 3: grow_body<E, 3, false, REAL, false, NT>(ob, op.off0, op.off1, psi, nullptr, nullptr, first, step, e, sm.g); break;
        case 4: grow_body<E, 4, false, REAL, false, NT>(ob, op.off0, op.off1, psi, nullptr, nullptr, first, step, e, sm.g); break;
        default: break;
        }
        break;
    case BOP_GROW_ADJ:
        switch (op.R) {
        case 0: grow_body<E, 0, true, REAL, false, NT>(ob, op.off0, op.off1, psi, lam, gr, first, step, e, sm.g); break;
        case 1: grow_body<E, 1, true, REAL, false, NT>(ob, op.off0, op.off1, psi, lam, gr, first, step, e, sm.g); break;
        case 2: grow_body<E, 2, true, REAL, false, NT>(ob, op.off0, op.off1, psi, lam, gr, first, step, e, sm.g); break;
        case 3: grow_body<E, 3, true, REAL, false, NT>(ob, op.off0, op.off1, psi, lam, gr, first, step, e, sm.g); break;
        default: break;
        }
        break;
    case BOP_LAMBDA:
        lambda_body<E, NT>(psi, lam, b, e, reinterpret_cast<const TermDev *>(ob + op.off0), op.aux,
                           energies + op.energy, sm.l);
        break;
    case BOP_DIAG_ADJ:
        diag_adj_body<E, NT>(psi, lam, b, e, reinterpret_cast<const AdjDiagGate *>(ob + op.off0),
                      reinterpret_cast<const uint32_t *>(ob + op.off1), op.aux,
                      reinterpret_cast<const E *>(ob + op.off2), gr, sm.d);
        break;
    default: break;
    }
}

// NT threads per CTA, 2048 / NT... resident CTAs per SM at 128 registers: 16 warps
// per SM whatever NT is.
template <typename E, bool REAL, int NT>
__global__ void __launch_bounds__(NT, 512 / NT) batch_kernel(const uint8_t *__restrict__ blob,
                                                             const BatchOp *__restrict__ ops,
                                                             const BatchTask *__restrict__ tasks, uint32_t ntasks,
                                                             uint32_t *next, uint32_t *remaining, E *arena,
                                                             double *grads, double *energies, DevStatus *status,
                                                             long long spin_limit)
{
    __shared__ BatchShared<E, NT> sm;
    __shared__ uint32_t s_task, s_abort;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            s_task = atomicAdd(next, 1u);
            s_abort = 0;
        }
        __syncthreads();
        const uint32_t t = s_task;
        if (t >= ntasks) break;
        const BatchTask task = tasks[t];
        const BatchOp op = ops[task.op];
        if (op.dep != kNoDep && threadIdx.x == 0) {
            const long long t0 = clock64();
            while (*reinterpret_cast<volatile uint32_t *>(&remaining[op.dep]) != 0u) {
                if (clock64() - t0 > spin_limit) {
                    report(status, kErrTimeout, 100 + op.kind, t);
                    s_abort = 1;
                    break;
                }
                __nanosleep(128);
            }
            __threadfence();
        }
        __syncthreads();
        if (s_abort) break;
        const bool grow = op.kind == BOP_GROW || op.kind == BOP_GROW_ADJ;
        run_op_slice<E, REAL, NT>(op, blob, arena, grads, energies, task.begin, task.end, grow ? task.begin : 0,
                                  grow ? uint64_t(NT / 32) : 0, sm);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) atomicSub(&remaining[task.op], 1u);
    }
}

template <typename E, bool REAL, int NT>
cudaError_t persistent_typed(const uint8_t *blob, const BatchOp *ops, const BatchTask *tasks, uint32_t ntasks,
                             uint32_t *next, uint32_t *remaining, E *arena, double *grads, double *energies,
                             DevStatus *status, long long spin_limit, int sms, cudaStream_t st)
{
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<E, REAL, NT>, NT, 0);
    if (per_sm < 1) per_sm = 1;
    batch_kernel<E, REAL, NT><<<unsigned(sms * per_sm), NT, 0, st>>>(blob, ops, tasks, ntasks, next, remaining, arena,
                                                                     grads, energies, status, spin_limit);
    return cudaGetLastError();
}

template <typename E, bool REAL>
cudaError_t persistent_threads(int threads, const uint8_t *blob, const BatchOp *ops, const BatchTask *tasks,
                               uint32_t ntasks, uint32_t *next, uint32_t *remaining, E *arena, double *grads,
                               double *energies, DevStatus *status, long long spin_limit, int sms, cudaStream_t st)
{
    switch (threads) {
    case 64:
        return persistent_typed<E, REAL, 64>(blob, ops, tasks, ntasks, next, remaining, arena, grads, energies,
                                             status, spin_limit, sms, st);
    case 128:
        return persistent_typed<E, REAL, 128>(blob, ops, tasks, ntasks, next, remaining, arena, grads, energies,
                                              status, spin_limit, sms, st);
    case 256:
        return persistent_typed<E, REAL, 256>(blob, ops, tasks, ntasks, next, remaining, arena, grads, energies,
                                              status, spin_limit, sms, st);
    default: return cudaErrorInvalidValue;
    }
}

template <typename E>
cudaError_t persistent_real(bool real, int threads, const uint8_t *blob, const BatchOp *ops, const BatchTask *tasks,
                            uint32_t ntasks, uint32_t *next, uint32_t *remaining, E *arena, double *grads,
                            double *energies, DevStatus *status, long long spin_limit, int sms, cudaStream_t st)
{
    return real ? persistent_threads<E, true>(threads, blob, ops, tasks, ntasks, next, remaining, arena, grads,
                                              energies, status, spin_limit, sms, st)
                : persistent_threads<E, false>(threads, blob, ops, tasks, ntasks, next, remaining, arena, grads,
                                               energies, status, spin_limit, sms, st);
}

}  // namespace

cudaError_t run_batch_persistent(const uint8_t *blob, const BatchOp *ops, const BatchTask *tasks, uint32_t ntasks,
                                 uint32_t *next, uint32_t *remaining, void *arena, double *grads, double *energies,
                                 DevStatus *status, int elem_bytes, bool real, int threads, int wait_limit_log2,
                                 int sms, cudaStream_t st)
{
    const long long spin_limit = 1LL << wait_limit_log2;
    if (elem_bytes == 8)
        return persistent_real(real, threads, blob, ops, tasks, ntasks, next, remaining, static_cast<float2 *>(arena),
                               grads, energies, status, spin_limit, sms, st);
    return persistent_real(real, threads, blob, ops, tasks, ntasks, next, remaining, static_cast<double2 *>(arena),
                           grads, energies, status, spin_limit, sms, st);
}

}  // namespace zxh
