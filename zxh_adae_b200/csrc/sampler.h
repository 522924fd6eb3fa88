// sampler.h -- device scratch layout and launcher of the multinomial sampler.
#pragma once

#include "core.h"

#include <cuda_runtime.h>

namespace zxh {

struct SamplerScratch {
    double *segcdf = nullptr;
    uint32_t *heavy_count = nullptr;
    void *flags_begin = nullptr, *flags_end = nullptr;  // region zeroed before every draw
    unsigned long long *counts = nullptr, *offsets = nullptr, *bsum = nullptr;
    uint32_t *heavy_list = nullptr;
    uint64_t *real = nullptr, *words = nullptr;
    uint64_t *coltab = nullptr;
    double *parts = nullptr;  // optional: the 32 lane-range masses of every segment

    static size_t need_bytes(uint64_t nseg, uint64_t shots, bool parts = false);
    void carve(uint8_t *base, uint64_t nseg, uint64_t shots, bool parts = false);
};

uint64_t mix_seed_host(uint64_t base, uint64_t salt);

// Draws shots outcomes from the 2^m-amplitude state into sc.real (real indices,
// grouped by segment) and sc.words (virtual bits, one word per shot for n <= 63).
cudaError_t run_sampler(const void *state, int elem_bytes, int m, uint64_t shots, uint64_t stream_seed,
                        const uint64_t *host_coltab, uint64_t b, SamplerScratch &sc, DevStatus *status, int sms,
                        cudaStream_t st, uint64_t &kernels);

// Counts of the draw left in sc by run_sampler on a 2^m-amplitude state (map
// offset b): pass 1 writes every segment's number of distinct outcomes (nuniq),
// their exclusive scan (uoff) and the total; pass 2 writes the distinct outcomes'
// virtual words and counts at uoff, in increasing real index.
cudaError_t run_counts(const SamplerScratch &sc, int m, uint64_t b, unsigned long long *nuniq,
                       unsigned long long *uoff, unsigned long long *total, uint64_t *words, uint64_t *hits,
                       int pass, int sms, cudaStream_t st, uint64_t &kernels);

// run_sampler's draw up to real indices, into a caller buffer (noalloc.cu).
cudaError_t run_sampler_real(const void *state, int elem_bytes, int m, uint64_t shots, uint64_t stream_seed,
                             uint64_t *real_out, SamplerScratch &sc, DevStatus *status, int sms, cudaStream_t st);

// Pass runner and get_state scatter (kernels.cu).
struct Pass;
// first_src / last_dst (only where the first / last pass is a general strided
// pass): that pass reads psi from first_src / writes it to last_dst instead of
// working on state in place.
cudaError_t run_passes(const std::vector<Pass> &passes, const uint8_t *dblob, void *state, int elem_bytes,
                       DevStatus *status, int sms, cudaStream_t st, uint64_t &kernels, const void *first_src = nullptr,
                       void *last_dst = nullptr);
// prefetch: each warp stages the next tile in shared memory with a TMA bulk copy
// while it works on the current one (waits bounded; a timeout sets status).
cudaError_t run_diag(const uint8_t *dblob, uint64_t doff, uint64_t toff, int m, int elem_bytes, int row_bits,
                     int chunk_bits, bool prefetch, void *state, DevStatus *status, int sms, cudaStream_t st);
int diag_tile_bits(int elem_bytes, int row_bits);
// The diagonal window as a Walsh sum (walsh.cu): one pass, cost per amplitude
// independent of the window's size and of the affine map; needs m >= walsh_tile_bits.
// n_terms: the compiled window's term count (sizes the shared-memory stage).
cudaError_t run_walsh(const uint8_t *dblob, uint64_t woff, uint64_t toff, int m, uint32_t n_terms, int elem_bytes,
                      void *state, int sms, cudaStream_t st);
int walsh_tile_bits(int elem_bytes);
cudaError_t run_fast_tile(const uint8_t *dblob, uint64_t foff, uint64_t toff, uint64_t ntiles, int elem_bytes,
                          void *state, DevStatus *status, int sms, cudaStream_t st);
// low: the low pass (lane bits swapped into registers); real: every gate of the
// pass has a real matrix (both need row_low_ok); win: the pass has a window.
cudaError_t run_row_pass(const uint8_t *dblob, uint64_t poff, uint64_t toff, uint64_t nitems, int elem_bytes,
                         int wide, bool low, bool real, bool win, void *state, int sms, cudaStream_t st);
// Span pass (span.cu): up to T real-rotation gates on a 2^T-amplitude tile per
// read-modify-write (T = 13 complex64, 12 complex128); low: the tile is real bits
// 0..T-1; layouts: 2 or 3 (span_layouts); land: the landing form; win: 0 no window,
// 1 windows with linear terms only, 2 windows with quadratic terms; rot, pos: the
// pass's rotation coefficients and tile coordinates (host copies of SpanDev::rot and
// SpanDev::pos, passed to the landing form as a kernel parameter).
cudaError_t run_span(const uint8_t *dblob, uint64_t soff, uint64_t toff, uint64_t ntiles, int elem_bytes, bool low,
                     int layouts, bool land, int win, void *state, const double (*rot)[2], const uint8_t *pos, int sms,
                     cudaStream_t st);
// amplitude 0 := 1 (the rest of an INIT pass is a memset)
cudaError_t run_set_one(void *state, int elem_bytes, cudaStream_t st);
// General strided pass (grow.cu): lam == nullptr applies the pass to psi; otherwise
// the adjoint form on psi and lam with gradients added to grads[slot]. real: every
// gate of the pass has a real matrix (GrowBuild::all_real). staged: the form whose
// warps copy their next item into shared memory during the current one (needs
// status, where a wait that gives up is recorded).
// psi_src: read psi from there (written to psi).
cudaError_t run_grow(const uint8_t *dblob, uint64_t poff, uint64_t toff, int R, uint64_t nitems, int elem_bytes,
                     void *psi, void *lam, double *grads, bool real, bool staged, DevStatus *status, int sms,
                     cudaStream_t st, const void *psi_src = nullptr);
int grow_reg_bits(int elem_bytes, bool adjoint);
int grow_fixed_bits(int elem_bytes);
int grow_adjoint_gates();
cudaError_t run_scatter(const void *state, uint64_t n_real, const uint64_t *dcoltab, uint64_t b, int N, int order,
                        double gre, double gim, void *out, int elem_bytes, int sms, cudaStream_t st);

}  // namespace zxh
