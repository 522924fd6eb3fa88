/*
 * zxh_oracle.h -- TEST INFRASTRUCTURE ONLY. A plain-C, single-threaded CPU
 * restatement of ZXH-Sim's single-GPU execute()/measure()/get_state() path, used
 * as the checker for the CUDA product. Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it; the product never links it.
 *
 * Pinned against the reference itself: tests compare it with the unmodified
 * reference compiled from source (oracle/_ref/libzxhref_*.so) and with the
 * committed golden fixtures under tests/golden/.
 */
#ifndef ZXH_ORACLE_H
#define ZXH_ORACLE_H

#include <stddef.h>
#include <stdint.h>

typedef struct zxo_sim zxo_sim;

/* Records use the 40-byte zxh_gate layout of include/zxh_b200.h. */
zxo_sim *zxo_create(int n, int disable_x, int eager_expand_all);
void zxo_destroy(zxo_sim *s);
int zxo_push(zxo_sim *s, const void *recs, size_t count);
int zxo_clear_gates(zxo_sim *s);
int zxo_execute(zxo_sim *s);
size_t zxo_required_M(zxo_sim *s);
/* 2^n complex128 (interleaved); order 0 = reference (bit-reversed), 1 = qubit order. */
int zxo_get_state(zxo_sim *s, double *out, int order);
/* Real-address state, 2^m complex128, without the global phase. */
int zxo_real_state(zxo_sim *s, double *out, size_t *m_out);
void zxo_global_phase(zxo_sim *s, double *re, double *im);
/* Affine map after execute: rows[q] = alpha_q (m bits), b bit q. */
int zxo_affine(zxo_sim *s, uint64_t *rows, uint64_t *b, size_t *m_out);
/* Restates the reference GPU sampler (measure_cuda.cu): words = ceil(n/64) per shot;
 * real_out (may be NULL) gets the real index of each shot in output order. */
int zxo_sample_gpu(zxo_sim *s, uint64_t seed, size_t shots, uint64_t *words, uint64_t *real_out);
/* The sampler's uniform for one draw: stream 0 picks the segment by shot index,
 * stream 1 picks the offset by output index (measure_cuda.cu:395-410,427,498). */
double zxo_uniform(uint64_t seed, int stream, uint64_t idx);

#endif
