// core.h -- host-side types of the B200-native ZXH path: gate records, the GF(2)
// affine address map, the operation list produced by the execute() walk, and the
// per-pass programs handed to the device kernels.
//
// Reference: ZXH-Sim (AxEquals-b/ZXH_ADAE), src/zxh/. The affine map follows
// src/core/bitmat.cpp:34-161 and selector.cpp:20-49; the walk follows
// src/core/zxh.cpp:312-553.
#pragma once

#include <complex>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace zxh {

using cd = std::complex<double>;

enum GateType : uint32_t {
    G_NONE = 0,
    G_BARRIER = 1,
    G_Z = 2,
    G_RZ = 3,
    G_P = 4,
    G_CRZ = 5,
    G_CP = 6,
    G_X = 7,
    G_CX = 8,
    G_H = 9,
    G_U3 = 10,
    G_RX = 11,
};

struct Gate {
    uint32_t type;
    uint32_t cq;
    uint32_t q;
    uint32_t reserved;
    double theta;
    double lambda;
    double phi;
};
static_assert(sizeof(Gate) == 40, "gate record is 40 bytes");

// A selector S(x) = parity(alpha & x) xor beta over real addresses
// (src/zxh/include/zxhsim/defs.h:23-37).
struct Sel {
    uint64_t alpha = 0;
    int beta = 0;
};

inline int parity64(uint64_t x) { return __builtin_popcountll(x) & 1; }
inline uint64_t low_mask(int bits) { return bits >= 64 ? ~0ULL : ((1ULL << bits) - 1ULL); }

// GF(2) affine map x_virtual = A x_real xor b. rows[q] is row q of A (m bits).
// Columns are linearly independent, so A x = e_q has at most one solution. All
// solutions are computed at once by one elimination of [A | I] and cached until the
// map changes (the reference re-runs a full elimination for every U3 probe,
// bitmat.cpp:46-122).
class AffineMap {
  public:
    void reset(int n);
    int n() const { return n_; }
    int m() const { return m_; }
    uint64_t row(int q) const { return rows_[q]; }
    uint64_t b() const { return b_; }
    Sel selector(int q) const { return Sel{rows_[q], int((b_ >> q) & 1)}; }
    // delta with A delta = e_q; false if e_q is outside the column span.
    bool solve(int q, uint64_t &delta);
    void append_col(int q);          // append e_q as a new column
    void row_xor(int dst, int src);  // CX transport
    void flip_b(int q) { b_ ^= 1ULL << q; }
    void b_xor(int dst, int src) { if ((b_ >> src) & 1) b_ ^= 1ULL << dst; }
    // virtual index of a real index
    uint64_t virt(uint64_t real) const;

  private:
    void refresh();
    int n_ = 0;
    int m_ = 0;
    uint64_t rows_[64] = {0};
    uint64_t b_ = 0;
    bool dirty_ = true;
    uint64_t sol_[64] = {0};
    uint64_t solvable_ = 0;
};

// ---------------------------------------------------------------------------
// Operation list: what the reference's execute() would launch, in order, with
// real-address selectors and deltas already resolved.

struct U3Op {
    uint64_t delta = 0;
    Sel sel;            // pair (i, i^delta) with S(i) == 0 is "even"
    cd u[4];            // u00, u01, u10, u11
    bool has_ctrl = false;
    Sel ctrl;           // explicit CX: act only where ctrl(i) == 1
};

struct DiagTerm {
    Sel s0, s1;
    bool two = false;   // CP (s0 && s1) vs P (s0)
    double theta = 0.0;
};

struct Op {
    enum Kind { EXPAND, U3BATCH, DIAG } kind;
    // EXPAND: state grows from m to m+1 bits then one pair op with delta 2^m.
    // U3BATCH: pair ops applied in order on the current 2^m block.
    // DIAG: one diagonal window.
    int m = 0;                   // state bits when the op runs (after growth for EXPAND)
    std::vector<U3Op> u3;
    std::vector<DiagTerm> diag;
};

// ---------------------------------------------------------------------------
// Device programs (plain-old-data, uploaded once per execute()).

constexpr int kMaxTileBits = 16;

struct LinTerm { uint32_t bit; uint32_t pad; int64_t coef; };
struct QuadTerm { uint32_t i; uint32_t j; int64_t coef; };
struct GenTerm {
    uint64_t a1_t, a1_out, a2_t, a2_out;  // selector masks split into tile coords / out-of-tile real bits
    uint32_t b1, b2;
    int64_t coef;                         // added where S1 && S2 (P: S2 == 1 always)
};

// One diagonal window compiled for a tile geometry. Phases are int64 fixed-point
// turns: coef / 2^64 of a full turn, so sums wrap exactly modulo 2*pi.
struct DiagDev {
    int64_t c0;
    int64_t lin_in[kMaxTileBits];   // linear coefficient of each tile coordinate
    uint32_t n_out_lin, n_out_quad, n_in_quad, n_cross, n_gen, pad;
    uint64_t off_out_lin, off_out_quad, off_in_quad, off_cross, off_gen;  // byte offsets in the blob
    uint64_t off_kidx;  // uint32[kMaxTileBits + 1]: cross terms are sorted by tile coordinate i,
                        // those of coordinate k are [kidx[k], kidx[k+1])
};

// A diagonal window as a Walsh sum (walsh.cu): phase(r) = c0 + sum over terms of
// w * (-1)^parity(mask & r), every term's mask split into its in-tile part g (the
// low T bits) and out-of-tile part hi (mask >> T). hi_g packs hi (bits 0..53: m <=
// 63 and T >= 9) with g above it (bits 54..63). Terms are sorted by g. Phases are
// int64 fixed-point turns (wrapping modulo 2^64 = one turn).
constexpr int kWalshGShift = 54;
struct WalshTermDev { uint64_t hi_g; int64_t w; };
struct WalshDev {
    int64_t c0;
    uint32_t T, n_terms;
    uint64_t off_terms;  // byte offset of WalshTermDev[n_terms] in the blob
};

// exp(2 pi i j / 1024), j = 0..1023: the coarse factor of a phase given in turns.
constexpr int kExpTableBits = 10;

struct U3Dev {
    uint64_t delta_t;   // delta in tile coordinates
    uint64_t alpha_t;   // selector alpha restricted to tile coordinates
    uint64_t alpha_out; // selector alpha on out-of-tile real bits
    uint32_t beta;
    uint32_t pivot;     // a set bit of delta_t
    uint64_t ctrl_t, ctrl_out;
    uint32_t ctrl_beta, has_ctrl;
    double u[8];        // u00 re,im, u01, u10, u11
};

struct StepDev { uint32_t kind; uint32_t pad; uint64_t off; };  // kind 0 = DIAG, 1 = U3
enum { STEP_DIAG = 0, STEP_U3 = 1 };

// Tile geometry: tile coordinate k maps to real bit pos[k]. Coordinates [0, c) are
// the c low contiguous bits; coordinates [c, T) are single high bits.
struct TileDev {
    uint32_t T, c, h, m;
    uint64_t tile_mask;   // real bits inside the tile
    uint64_t free_mask;   // real bits < m outside the tile (tile index deposits here)
    uint64_t ntiles;
    uint8_t pos[kMaxTileBits];
    uint32_t nsteps, pad;
    uint64_t off_steps;
};

struct ExpandDev {
    uint32_t m_old;      // doubling from 2^m_old to 2^(m_old+1)
    uint32_t has_ctrl;
    uint64_t alpha;      // selector of the pair op restricted to old bits
    uint32_t beta, ctrl_beta;
    uint64_t ctrl_alpha;
    double u[8];
};

// A pair op applied straight in global memory (deltas spanning more high bits
// than a tile holds).
struct PairDev {
    uint32_t m, pivot;
    uint64_t delta, alpha;
    uint32_t beta, has_ctrl;
    uint64_t ctrl_alpha;
    uint32_t ctrl_beta, pad;
    double u[8];
};

// Product state written in one pass: amplitude(y) = L[y low c0 bits] *
// M[next c1 bits] * H[remaining c2 bits] (the initial amplitude folded into H).
// The three tables follow each other in the blob at off2.
struct ProductDev {
    uint32_t m, c0, c1, c2;
};

// Fast tile pass (u3pass.cu): every pair op has a single-bit delta equal to its
// selector bit (the X-transported map is a permutation on those bits) and no
// control. Tile coordinates 0..4 are the lanes of a warp; per shared-memory round
// R coordinates are held in registers and 3 more select the warp.
constexpr int kFastMaxGates = 16;
constexpr int kFastMaxRounds = 4;

struct FastGateDev {
    uint32_t coord;      // tile coordinate of the gate's bit
    uint32_t round;      // register round the gate runs in (lane gates: round 0)
    uint64_t alpha_out;  // selector bits outside the tile (tile parity flips beta)
    uint32_t beta, pad;
    double u[8];
};

struct RoundDev {
    uint8_t rc[4];  // register coordinates
    uint8_t oc[3];  // warp coordinates
    uint8_t pad;
};

struct FastDev {
    TileDev g;
    uint32_t R, nrounds, ngates, pad;
    RoundDev rounds[kFastMaxRounds];
    uint64_t off_gates;
    uint64_t off_pre, off_post;  // DiagDev offsets of the fused windows, 0 if none
};

// Strided high-qubit pass (u3pass.cu): real bits [0, F) are a thread's 16-byte
// vector and the lanes of its warp (F = 6 for complex64, 5 for complex128); R more
// bits (the gates' bits, any positions) are a thread's registers; every other bit
// enumerates work items. Each register row of a warp is 512 contiguous bytes and
// the warps of a CTA take consecutive items.
struct RowPassDev {
    uint32_t m, F, R, ngates;
    uint8_t rb[8];        // real bits of the register coordinates, ascending
    uint64_t tile_mask;   // bits [0, F) and rb
    uint64_t nitems;      // 2^(m - F - R)
    uint64_t off_gates;   // FastGateDev[ngates] (coord = tile coordinate, round unused)
    uint64_t off_pre, off_post;
};

// Span pass (span.cu): a CTA holds a tile of 2^T amplitudes (T = 13 complex64, 12
// complex128) whose coordinates k = 0..T-1 are the real bits pos[k] (ascending: bits
// 0..c-1, then the gates' bits); every other real bit enumerates tiles. The
// amplitudes move between register layouts through shared memory, so a gate on any
// coordinate is a register update: one pass applies up to T gates (the low pass,
// c = T) or up to T - 3 on high bits (c >= 3). Coordinate k's real rotation [[c, -s], [s, c]]
// (already oriented by its selector's beta) is stored with one coefficient
// factored out: rot[k] = (tau, 0) with tau = s / c when |c| >= |s| (x' = x - tau y,
// y' = y + tau x, factor c), else (mu, 1) with mu = c / s (x' = mu x - y,
// y' = x + mu y, factor s). scale is the product of the factors of all the pass's
// gates: the same for every amplitude, applied once.
constexpr int kSpanBits = 13;
struct SpanDev {
    uint32_t m, c, low, gates;  // low: the tile is real bits 0..12; gates: bit k = coordinate k has one
    uint8_t pos[16];
    uint64_t tile_mask, ntiles;
    double rot[kSpanBits][2];  // complex64 passes round both to float
    double scale;
    uint64_t off_pre, off_post;  // DiagDev windows (tile coordinates = pos), 0 if none
};

// General strided pass (grow.cu): like RowPassDev, but the R register
// coordinates are arbitrary pair deltas (several bits each, as after CX
// transport). A thread's row k holds the amplitudes at r0 ^ D[k] ^ (lane, vector)
// with D[k] = xor of delta_i over the set bits i of k; items r0 enumerate the
// addresses with zeros at bits [0, F) and at the pivot bits of the deltas'
// high parts. Gates whose delta lies inside [0, F) are lane gates (partner by
// shfl.xor / vector slot). Selectors are evaluated as parity(alpha & r0) (one
// per lane, ballot) xor a per-thread lane part; a gate's own selector depends on
// the row only through its own register coordinate.
constexpr int kGrowMaxSel = 64;
constexpr int kGrowMaxGates = 16;
constexpr int kGrowMaxTerms = 128;

struct GrowGateDev {
    uint32_t kind;    // 0: register coordinate `reg`; 1: lane gate
    uint32_t reg;
    uint32_t lane_x;  // lane gate: partner lane xor
    uint32_t vec_x;   // lane gate: partner vector-slot xor (complex64)
    uint32_t sel;     // index of the gate's selector
    uint32_t gen;     // adjoint passes: gradient generator (0 none, 1 Y, 2 X)
    uint32_t slot;    // adjoint passes: gradient slot
    uint32_t pad;
    double u[8];      // u00, u01, u10, u11 (re, im); adjoint passes hold U^dagger
};

struct GrowSelDev {
    uint64_t alpha;
    uint32_t beta;
    int32_t kbit;     // register coordinate the selector flips with, -1 if none
};

// One window term: phase coef (64-bit turns) where selector s0 (and s1 unless
// s1 == 0xff) is 1. In adjoint passes coef is the inverse phase and the term's
// gradient sum_r Im(conj(lambda_r) psi_r) * (S(r) ? m1 : m0) goes to grads[slot]
// (gk 1: RZ, m0 = 1, m1 = -1; gk 2: P or CP, m0 = 0, m1 = -2; gk 0: none).
struct GrowTermDev {
    uint8_t s0, s1;
    uint8_t gk, pad;
    uint32_t slot;
    int64_t coef;
};

struct GrowDev {
    uint32_t m, F, R, ngates;
    uint64_t D[16];
    uint8_t piv[4];          // pivot bits, ascending
    uint32_t nsel;
    uint32_t ncls[2][3];     // pre / post window: end of class 0 (one selector, no row dependence),
                             // end of class 1 (two selectors, no row dependence), total terms
    uint64_t nitems;
    uint64_t off_gates, off_sel;
    uint64_t off_terms[2];
};

// Status word shared with the device (bounded waits report here).
struct DevStatus { uint32_t code; uint32_t where; uint64_t info; };

}  // namespace zxh
