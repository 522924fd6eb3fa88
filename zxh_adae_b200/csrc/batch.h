// batch.h -- the batched launch: many independent circuits, each a chain of
// passes over its own state, run by one persistent kernel (batch.cu) that takes
// tasks from a queue in order; a task waits until the previous pass of its
// circuit has finished.
#pragma once

#include "adjoint.h"
#include "core.h"

#include <cuda_runtime.h>

#include <cstdint>

namespace zxh {

enum BatchOpKind : uint32_t {
    BOP_INIT = 0,      // psi := |0...0>
    BOP_GROW = 1,      // general strided pass on psi
    BOP_LAMBDA = 2,    // lambda := H psi, energy += <psi|H|psi>
    BOP_GROW_ADJ = 3,  // general strided adjoint pass on psi and lambda, gradients
    BOP_DIAG_ADJ = 4,  // adjoint diagonal group on psi and lambda, gradients
};

constexpr uint32_t kNoDep = 0xffffffffu;
constexpr int kBatchDiagMax = 16;  // diagonal gates per adjoint group in the batch kernel (registers)

struct BatchOp {
    uint32_t kind, R, circuit, dep;  // dep: index of the op this one waits for
    uint64_t units;                  // items (grow passes) or amplitudes
    uint64_t base;                   // this op's descriptors start at blob + base
    uint64_t off0, off1, off2;       // GROW*: pass descriptor, phase table; LAMBDA: terms;
                                     // DIAG_ADJ: gates, slots, phase table (all from base)
    uint32_t aux, m;                 // LAMBDA: terms; DIAG_ADJ: gates; GROW*: 1 if every gate is real; m: state bits
    uint64_t psi, lam;               // element offsets of the circuit's states in the arena
    uint32_t grad_base, energy;      // the circuit's first gradient slot and its energy slot
};

struct BatchTask {
    uint32_t op, pad;
    uint64_t begin, end;  // units of the op
};

// Runs every task of the queue; counters: `next` (queue head, zeroed) and
// `remaining[op]` (tasks of each op, preset). grid = resident CTAs. real: every
// strided op of the queue has real gates (the kernel's real-gate form). threads:
// 64, 128 or 256 per CTA (the warps that work on one task). A task waits at most
// 2^wait_limit_log2 SM clocks for its op's predecessor; then it records a timeout
// in the status word and its CTA ends.
cudaError_t run_batch_persistent(const uint8_t *blob, const BatchOp *ops, const BatchTask *tasks, uint32_t ntasks,
                                 uint32_t *next, uint32_t *remaining, void *arena, double *grads, double *energies,
                                 DevStatus *status, int elem_bytes, bool real, int threads, int wait_limit_log2,
                                 int sms, cudaStream_t st);

}  // namespace zxh
