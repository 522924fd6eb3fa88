// host.h -- walk and planner interfaces (implemented in host.cpp).
#pragma once

#include "core.h"

namespace zxh {

struct WalkState {
    AffineMap map;
    int m = 0;                 // current real address bits of the state
    cd gphase = cd(1.0, 0.0);  // accumulated Z/Rz global phase (zxh.cpp:477-493)
    bool fresh = true;         // state is |0...0> and no device work has been done yet
    int init_bits = 0;         // bits of the fresh |0...0> state (n under eager_expand_all, else 0)
};

// Runs the reference execute() schedule over gates, updating ws (affine map, m,
// global phase) and appending the operations the reference would launch.
// M bounds the state size. Returns 0 or a status code with err set.
int walk(const Gate *gates, size_t count, bool disable_x, int M, WalkState &ws, std::vector<Op> &ops,
         std::string &err);

// U3(theta, lambda, phi) as the walk builds it (build_u3_matrix, zxh.cpp:101-113):
// u00, u01, u10, u11.
void u3_matrix(double theta, double lambda, double phi, cd u[4]);

// theta / (2 pi) as a 64-bit fixed-point fraction of a turn (wraps modulo 2^64).
int64_t phase_turns(double theta);
// exp(2 pi i j / 2^kExpTableBits), j = 0..1023, as complex64 or complex128 bytes.
void exp_table(int elem_bytes, std::vector<uint8_t> &bytes);

// calc_mem (zxh.cpp:648-681): real address bits the gate list needs.
int calc_mem(const Gate *gates, size_t count, int n, bool disable_x);

struct PlanParams {
    int tile_bits_c64 = 12;     // log2 amplitudes per TMA tile, complex64
    int tile_bits_c128 = 11;    // same for complex128
    int contig_bits = 6;        // contiguous low bits of a tile that also spans high bits
    int max_gates = 12;         // pair ops per generic tile pass
    int fast_gates = 6;         // fused gates per TMA low-qubit pass (bounded by the FMA budget per byte)
    int fast_fuse_quad = 32;    // largest in-tile quadratic term count of a window fused into a fast pass
    int fast_contig_c64 = 4;    // contiguous low bits of a fast tile that also spans high bits (complex64)
    int fast_contig_c128 = 3;   // same for complex128
    int row_wide_c64 = 1;       // strided pass shape, complex64: 0 = 16-byte lanes x 16 rows (4 register bits),
                                // 1 = 8-byte lanes x 32 rows (5 register bits: a 30-qubit U3 layer in 5 passes)
    int row_wide_c128 = 1;      // complex128: 0 = 8 rows, 1 = 16 rows
    int low_pass = 1;           // 1: gates on the lane / vector bits ride in a strided low pass (lane bits
                                // swapped into registers) instead of the TMA fast pass
    int low_regs_c64 = 5;       // gates on register bits that join the low pass, complex64 (0..5; at most
                                // the shape's register bits)
    int low_regs_c128 = 4;      // same for complex128
    int real_split = 1;         // 1: in all-strided U3 batches each gate runs as a real rotation; its phases
                                // ride in the windows before / after the batch (half the multiply-adds)
    int max_steps = 16;
    int diag_row_bits_c64 = 2;  // log2 rows of a warp tile in a diagonal pass (tile = 64 amplitudes x rows:
                                // 2 KiB; with 32 KiB chunks 1.00 of measured HBM at 30-32 qubits on B200)
    int diag_row_bits_c128 = 3; // same for complex128 (tile = 32 amplitudes x rows: 4 KiB)
    int grow = 1;               // 1: U3 batches with multi-bit deltas use the general strided pass (grow.cu)
    int grow_regs = 4;          // register coordinates (gates with high deltas) per general strided pass
    int grow_only = 0;          // 1: only INIT and general strided passes (the persistent batch kernel's set)
    int adj_windows = 1;        // adjoint sweep: diagonal gates ride in the general strided passes as windows
    int adj_regs = 4;           // adjoint sweep: gates with high deltas per strided pass (4 runs at one CTA per SM)
    int grow_staged = 1;        // general strided passes whose warps stage their next item in shared memory
                                // (TMA bulk copies): bit 0 the adjoint sweep's in complex64, bit 1 the
                                // forward ones, bit 2 the adjoint sweep's in complex128 (measured on the
                                // 24-qubit ansatz: -2 % complex64 adjoint, +3 % complex128, +3 % forward)
    int diag_prefetch_c64 = 1;  // diagonal pass: each warp stages its next tile with a TMA bulk copy
    int diag_prefetch_c128 = 0; // same for complex128 (no gain measured there)
    int diag_chunk_bits = -1;   // log2 tiles a warp walks in Gray-code order in a diagonal pass (-1: as many
                                // as span 32 KiB)
    int product_table_bits = 12;
    int walsh = 1;              // 1: windows with multi-bit selectors run as one Walsh-sum pass (walsh.cu)
                                // instead of general terms evaluated per amplitude (split every 32 terms)
    int walsh_min_general = 2;  // general (multi-bit selector) terms from which a standalone window takes the
                                // Walsh pass; 0: every standalone window does
    int span = 1;               // U3 batches (real split) run as span passes (span.cu): the gates on bits
                                // 0..T-1 in one pass, then up to T - span_min_run high-bit gates per pass
                                // (T = 13 complex64, 12 complex128); 0: the register-row passes
    int span_land = 1;          // span passes in the landing form (the next tile lands in shared memory
                                // during the current one); 0: the register form
    int span_min_run = 3;       // log2 of the shortest run of contiguous amplitudes a strided span pass
                                // reads (3..8: 64 B .. 2 KiB complex64, 128 B .. 4 KiB complex128)
                                // (3: a 32-qubit layer in 3 passes, 54.7 ms on B200, vs 4 passes, 57.2 ms)
    int span_split = 0;         // how the high-bit gates are dealt to the strided span passes: 0 in blocks of
                                // neighbouring bits, the larger blocks on the lower bits; 1 round robin (every
                                // pass gets bits from the whole range); 2 blocks, the larger on the higher bits
    int span_mixed = 1;         // 1: a U3 batch mixing single-bit and multi-bit pair deltas (at least 8
                                // single-bit gates) runs the single-bit gates as span passes first
    int span_order = 0;         // order of the strided span passes (the first one carries the window before the
                                // batch): 0 from the lowest bits up, but the first pass that runs two layouts
                                // (not three) moved to the front; 1 from the lowest bits up; 2 from the highest down
};

// General strided pass shape (grow.cu): fixed low bits and register coordinates.
int grow_reg_bits(int elem_bytes, bool adjoint);
int grow_fixed_bits(int elem_bytes);

// Builds the selector table and gate / window records of one general strided pass
// over register deltas `regs` (full real-address deltas) on a 2^m state. Returns
// false if a window's selector flips with more than one register coordinate or
// the tables overflow (the caller then runs the window on its own).
struct GrowBuild {
    int elem_bytes = 8, m = 0;
    std::vector<uint64_t> regs;
    GrowDev dev;
    std::vector<GrowGateDev> gates;
    std::vector<GrowSelDev> sels;
    std::vector<GrowTermDev> terms[2];
    bool init(int elem_bytes, int m, const std::vector<uint64_t> &regs);
    int selector(const Sel &s);  // -1 on overflow or a multi-coordinate flip
    bool add_gate(const U3Op &u, uint32_t gen, uint32_t slot, bool adjoint_matrix);
    // which: 0 before the gates, 1 after. Adjoint passes give per-term gradient
    // kinds and slots and inverse = true (the inverse phase is applied).
    bool add_window(int which, const std::vector<DiagTerm> &w, const std::vector<uint32_t> *gk = nullptr,
                    const std::vector<uint32_t> *slot = nullptr, bool inverse = false);
    bool all_real() const;  // every gate matrix has zero imaginary parts
};

struct Pass {
    enum Kind { PRODUCT, EXPAND, TILE, PAIR, DIAG, FAST, ROW, GROW, INIT, WALSH, SPAN } kind;  // INIT: |0...0> (grow_only)
    int m = 0;
    uint64_t off = 0;    // blob offset of the pass descriptor
    uint64_t off2 = 0;   // PRODUCT: lookup table; DIAG: exp table
    TileDev geom;        // TILE
    std::vector<StepDev> steps;
    FastDev fast;                        // FAST
    RowPassDev row;                      // ROW
    SpanDev span;                        // SPAN
    int wide = 0;                        // ROW: kernel shape
    int low = 0;                         // ROW: the low pass (lane bits 0..3 swapped into registers);
                                         // SPAN: the tile is real bits 0..12
    int real = 0;                        // ROW: every gate matrix is real; SPAN: its windows (0 none,
                                         // 1 linear terms only, 2 quadratic terms), set when the plan is done
    int chunk_bits = -1;                 // DIAG: tiles per Gray-code chunk (log2, -1 = automatic)
    int row_bits = 0;                    // DIAG: log2 rows of a warp tile; WALSH: the window's term count
    int prefetch = 0;                    // DIAG: tiles staged one ahead by TMA bulk copies; GROW: the
                                         // staged form (next item in shared memory); SPAN: the landing form
    std::vector<FastGateDev> fgates;     // FAST
    GrowBuild gb;                        // GROW
};

struct Plan {
    std::vector<uint8_t> blob;
    std::vector<Pass> passes;
    void clear();
};

// Tile bits of the standalone diagonal pass (diag.cu), of the Walsh-sum window
// pass (walsh.cu) and of the fast U3 pass (u3pass.cu), and the register bits of
// one fast-pass round.
int diag_tile_bits(int elem_bytes, int row_bits);
int walsh_tile_bits(int elem_bytes);
// Span pass (span.cu): tile coordinates (13 for complex64, 12 for complex128), and
// the register layouts a pass with the gates of `gates` (bit k = coordinate k) runs
// through (land: the complex64 landing form): 2 or 3, 0 if some gate sits on a
// coordinate no layout holds in registers.
int span_tile_bits(int elem_bytes);
int span_layouts(int elem_bytes, uint32_t gates, bool low, bool land);
int fast_tile_bits(int elem_bytes);
int fast_reg_bits(int elem_bytes);
int row_reg_bits(int elem_bytes, int wide);
int row_fixed_bits(int elem_bytes, int wide);
bool row_low_ok(int elem_bytes, int wide);  // the shape's lane bits can swap with its rows (the low pass)

// carry_in: phases due on the state before the ops (left over by the previous
// plan; real-bit selectors, so the affine map's changes since do not touch them);
// carry_out: if given, the phases split off the last U3 batch are returned there
// instead of being applied (the caller applies them later, or hands them to the
// next plan, whose first U3 batch takes them into its own window).
int plan(const std::vector<Op> &ops, int elem_bytes, const PlanParams &pp, const WalkState &start, Plan &out,
         std::string &err, const std::vector<DiagTerm> *carry_in = nullptr,
         std::vector<DiagTerm> *carry_out = nullptr);

}  // namespace zxh
