// adjoint.h -- device records and launchers of the expectation and adjoint-sweep
// kernels (adjoint.cu), shared with the host side (adjoint_api.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace zxh {

// One observable term in real-address form: Z_q is the selector
// parity(a0 & r) ^ b0, Z_q0 Z_q1 the xor of two selectors, X_q the flip r ^ delta.
struct TermDev {
    uint32_t kind, pad;  // ZXH_TERM_Z / ZZ / X
    uint64_t a0, a1;
    uint32_t b0, b1;
    uint64_t delta;
    double coef;
};

constexpr uint32_t kMaxTerms = 256;

// One 2x2 gate of the reverse sweep on pairs (r, r ^ delta); the member with
// selector parity(alpha & r) ^ beta == 0 is the |0> amplitude of the qubit.
struct AdjPairDev {
    uint32_t m, pivot;  // state bits; a set bit of delta
    uint64_t delta, alpha;
    uint32_t beta, gen; // generator of the gradient: 0 none, 1 Y (RY), 2 X (RX)
    double u[8];        // forward matrix u00, u01, u10, u11 (re, im); the kernel applies its adjoint
};

constexpr int kAdjDiagMax = 32;

// One diagonal gate of a commuting group: phase tq (64-bit turns) where the
// selector s (s0, or s0 and s1 when two = 1) is 1. Its gradient is
// sum_r Im(conj(lambda_r) psi_r) * (s(r) ? m1 : m0): RZ m0 = 1, m1 = -1 (Im<lambda|Z|psi>);
// P and CP m0 = 0, m1 = -2 (-2 Im<lambda|Pi_1|psi>); Z 0, 0.
struct AdjDiagGate {
    uint64_t a0, a1;
    uint32_t b0, b1;
    uint32_t kind, two;  // kind 0: no gradient
    int64_t tq;
    double m0, m1;
};

// lambda = H psi over 2^m amplitudes (lam may be null: energy only); adds
// <psi|H|psi> to *energy.
cudaError_t run_lambda(const void *psi, void *lam, int m, int elem_bytes, const TermDev *dterms, uint32_t nterms,
                       double *energy, int sms, cudaStream_t st);
// Adds Im<lam|G|psi> to *grad (gen != 0), then psi <- U^dagger psi, lam <- U^dagger lam.
cudaError_t run_adj_pair(void *psi, void *lam, int elem_bytes, const AdjPairDev &g, double *grad, int sms,
                         cudaStream_t st);
// For each gate j of the group adds its gradient to grads[slots[j]], then
// multiplies psi and lam by the inverse of the group's phase.
// gates and slots are HOST arrays of ng <= kAdjDiagMax entries, passed to the
// kernel by value (its constant bank); exp_tab: exp(2 pi i j / 1024) in the
// state's element type (device memory).
cudaError_t run_adj_diag(void *psi, void *lam, int m, int elem_bytes, const AdjDiagGate *gates, uint32_t ng,
                         double *grads, const uint32_t *slots, const void *exp_tab, int sms, cudaStream_t st);

}  // namespace zxh
