// adjoint_host.h -- host side of the adjoint sweep shared by the per-simulator
// entry points (adjoint_api.cpp) and the batched persistent launch (batch_api.cpp):
// observable compilation, the reverse program and its general strided passes.
#pragma once

#include "adjoint.h"
#include "sim.h"

#include <algorithm>
#include <string>
#include <vector>

namespace zxh {
namespace adj {

// Gradient generator of a lowered 2x2 record: 1 for RY = U3(theta, 0, 0), 2 for
// RX = U3(theta, pi/2, -pi/2), else 0.
uint32_t pair_generator(const Gate &g);
// RZ, P, CP, RY and RX records.
bool parameterised(const Gate &g);

// Observable terms in the real-address form of map A over m bits (errors are
// recorded on s).
int compile_terms(zxh_sim *s, const zxh_term *terms, size_t nterms, AffineMap &A, int m, bool drop_unreachable,
                  std::vector<TermDev> &out);

struct RevStep {
    enum Kind { PAIR, DIAG, RESTORE, GROW } kind;
    AdjPairDev pair;
    size_t slot = 0;   // PAIR: gradient slot
    size_t first = 0;  // DIAG: first gate in the uploaded group array
    uint32_t ng = 0;   // DIAG: gates in the group
    size_t ckpt = 0;   // RESTORE: checkpoint index
    zxh::GrowBuild gb; // GROW: commuting 2x2 gates on distinct qubits, adjoint form
    uint64_t off = 0;  // GROW: descriptor offset in the uploaded blob
    uint64_t toff = 0; // GROW: phase-table offset in the uploaded blob
};

// A run of 2x2 gates on distinct qubits with no CX between them, collected in
// reverse order; closed into one general strided adjoint pass (or single pair
// passes when the state is too small for one).
struct PairGroup {
    struct G {
        zxh::U3Op op;
        uint32_t gen;
        uint32_t slot;
        int q;
    };
    std::vector<G> gates;
    std::vector<uint64_t> basis;  // reduced high parts of the register deltas
    int nreg = 0;
    // Whether g can join (distinct qubit, room, independent high part).
    bool fits(const G &g, int F, int R, int m, int maxg) const
    {
        if (int(gates.size()) >= maxg) return false;
        for (const G &h : gates)
            if (h.q == g.q) return false;
        uint64_t hp = g.op.delta >> F;
        if (!hp) return true;
        if (nreg >= R || m < F + nreg + 1) return false;
        for (uint64_t b : basis)
            if ((hp >> (63 - __builtin_clzll(b))) & 1) hp ^= b;
        return hp != 0;
    }
    void add(const G &g, int F)
    {
        uint64_t hp = g.op.delta >> F;
        if (hp) {
            for (uint64_t b : basis)
                if ((hp >> (63 - __builtin_clzll(b))) & 1) hp ^= b;
            basis.push_back(hp);
            std::sort(basis.begin(), basis.end(), [](uint64_t a, uint64_t b) { return a > b; });
            nreg++;
        }
        gates.push_back(g);
    }
};


// Descriptors of the general strided adjoint passes, packed into one blob; sets
// each GROW step's offset.
std::vector<uint8_t> pack_grow(std::vector<RevStep> &steps);

// The reverse program of s->gates, walking the map back from A (the forward
// output's map, every qubit expanded); checkpoints end at ends[0..size-2].
int reverse_program(zxh_sim *s, const std::vector<size_t> &ends, AffineMap A, std::vector<RevStep> &steps,
                    std::vector<AdjDiagGate> &dgates, std::vector<uint32_t> &dslots, int diag_max = kAdjDiagMax);

}  // namespace adj
}  // namespace zxh
