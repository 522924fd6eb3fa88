/*
 * zxh_b200.h -- C ABI of the B200-native ZXH state-vector path.
 *
 * This is the drop-in boundary for ZXH-Sim's single-GPU circuit-run path: a gate
 * list goes in, the state, amplitudes or shot samples come out. Every entry point
 * takes plain pointers and sizes; no PyTorch or C++ type crosses it. Each call
 * returns ZXH_OK (0) or an error code; zxh_last_error() gives the message. No
 * entry point aborts the process (the reference calls std::abort on any error,
 * src/zxh/src/runtime/runtime_general.cpp:79-89).
 *
 * Citations are to the reference project ZXH-Sim (AxEquals-b/ZXH_ADAE), paths
 * relative to its root. The pybind11 surface these entry points replace is
 * src/zxh/src/pybind/bindings.cpp:79-118 (class _core.ZXH); the C++ methods behind
 * it are declared in src/zxh/include/zxhsim/zxh.h:11-53.
 */
#ifndef ZXH_B200_H
#define ZXH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Gate codes. Same numbering as the reference's gate_type_t
 * (src/zxh/include/zxhsim/defs.h:61-74). CRz is stored as P + CP and Rx as U3,
 * exactly as the reference records them (src/zxh/src/core/zxh.cpp:246-252,303-310). */
enum {
    ZXH_GATE_NONE = 0,
    ZXH_GATE_BARRIER = 1,
    ZXH_GATE_Z = 2,
    ZXH_GATE_RZ = 3,
    ZXH_GATE_P = 4,
    ZXH_GATE_CRZ = 5,
    ZXH_GATE_CP = 6,
    ZXH_GATE_X = 7,
    ZXH_GATE_CX = 8,
    ZXH_GATE_H = 9,
    ZXH_GATE_U3 = 10,
    ZXH_GATE_RX = 11 /* accepted by zxh_push_gates, recorded as U3(theta, pi/2, -pi/2) */
};

/* One gate record. Field meaning follows the reference's gate_t
 * (src/zxh/include/zxhsim/defs.h:76-84): U3 parameters are (theta, lambda, phi),
 * the order ZXH::U3 takes them (src/zxh/include/zxhsim/zxh.h:36). 40 bytes. */
typedef struct zxh_gate {
    uint32_t type;
    uint32_t cq;
    uint32_t q;
    uint32_t reserved;
    double theta;
    double lambda;
    double phi;
} zxh_gate;

/* Amplitude storage type of a simulator handle. The reference is complex128 only
 * (src/zxh/include/zxhsim/types.h:11-12); complex64 is this library's addition. */
enum { ZXH_C64 = 1, ZXH_C128 = 2 };

/* get_state orderings. ZXH_ORDER_REFERENCE is the reference's get_state order:
 * virtual index bit-reversed so qubit 0 is the most significant bit, times the
 * accumulated global phase (src/zxh/src/core/zxh.cpp:627-635). ZXH_ORDER_QUBIT
 * keeps qubit q at bit q (Qiskit order), also times the global phase. */
enum { ZXH_ORDER_REFERENCE = 0, ZXH_ORDER_QUBIT = 1 };

/* Status codes. */
enum {
    ZXH_OK = 0,
    ZXH_ERR_ARG = 1,     /* invalid argument (qubit out of range, null pointer, bad size) */
    ZXH_ERR_STATE = 2,   /* call out of order (e.g. get_state before execute) */
    ZXH_ERR_CUDA = 3,    /* CUDA runtime error */
    ZXH_ERR_OOM = 4,     /* device or host allocation failed */
    ZXH_ERR_LIMIT = 5,   /* size beyond a documented limit (n > 63, too many shots, ...) */
    ZXH_ERR_TIMEOUT = 6  /* a bounded device-side wait gave up */
};

typedef struct zxh_sim zxh_sim;

/* Library version string. */
const char *zxh_version(void);

/* Name (NUL-terminated, at most capacity - 1 characters) and SM count of CUDA
 * device `device`; either pointer may be NULL. Used to key tuned settings. No
 * counterpart in the reference. */
int zxh_device_info(int device, char *name, size_t capacity, int *sms);

/* Message of the last failing call on this handle, or of the last failing
 * zxh_create in this thread when sim is NULL. Never NULL. */
const char *zxh_last_error(const zxh_sim *sim);

/* Replaces ZXH::ZXH(N, disable_x, eager_expand_all) (zxh.h:14, zxh.cpp:209-212).
 * dtype is ZXH_C64 or ZXH_C128; device is the CUDA ordinal. n must be 1..63. */
int zxh_create(zxh_sim **out, size_t n, int disable_x, int eager_expand_all, int dtype, int device);
int zxh_destroy(zxh_sim *sim);

/* Replace ZXH::set_seed / clear_seed / clear_gates (zxh.cpp:216-232). */
int zxh_set_seed(zxh_sim *sim, uint64_t seed);
int zxh_clear_seed(zxh_sim *sim);
int zxh_clear_gates(zxh_sim *sim);

/* Per-gate recorders; replace ZXH::Barrier..ZXH::Rx (zxh.cpp:234-310). */
int zxh_barrier(zxh_sim *sim);
int zxh_rz(zxh_sim *sim, size_t q, double theta);
int zxh_crz(zxh_sim *sim, size_t cq, size_t q, double theta);
int zxh_cp(zxh_sim *sim, size_t cq, size_t q, double theta);
int zxh_p(zxh_sim *sim, size_t q, double theta);
int zxh_z(zxh_sim *sim, size_t q);
int zxh_x(zxh_sim *sim, size_t q);
int zxh_cx(zxh_sim *sim, size_t cq, size_t q);
int zxh_h(zxh_sim *sim, size_t q);
int zxh_u3(zxh_sim *sim, size_t q, double theta, double lambda, double phi);
int zxh_rx(zxh_sim *sim, size_t q, double theta);

/* Batch recorder: appends count records in one call (the reference's Python
 * loader calls one pybind method per gate, src/zxh/zxhsim/qasm.py:65-133).
 * Validates every record first; on error nothing is appended. */
int zxh_push_gates(zxh_sim *sim, const zxh_gate *gates, size_t count);

/* Replaces ZXH::execute (zxh.cpp:312-553): resets the state to |0...0>, runs the
 * whole recorded gate list on the device, and returns once the device is done. */
int zxh_execute(zxh_sim *sim);

/* Applies count more gates to the current state, continuing from where the last
 * zxh_execute / zxh_apply left the state and the affine map, without recording
 * them. Gates that would enlarge the state beyond the size chosen at the last
 * zxh_execute return ZXH_ERR_LIMIT. The phases that U3 gates leave after their
 * rotations (the real split's P(b) and global phase of the batch's last U3 gates)
 * are carried to the next zxh_apply, which takes them into the window before its
 * own first pass, so a circuit applied layer by layer costs what it costs in one
 * zxh_execute; every call that reads the state (zxh_measure, zxh_get_state*,
 * zxh_state_view, zxh_expectation) and zxh_flush apply them first. No counterpart
 * in the reference (its execute() always restarts from |0...0>,
 * zxh.cpp:329-338). */
int zxh_apply(zxh_sim *sim, const zxh_gate *gates, size_t count);

/* Applies the phases the last zxh_apply / zxh_apply_async carried over (one
 * diagonal pass; nothing when there are none) and returns once the device is
 * done; zxh_last_stats reports that pass. No counterpart in the reference. */
int zxh_flush(zxh_sim *sim);

/* zxh_apply without waiting: plans the batch on the host, queues its upload
 * (from one of two pinned program slots), its passes and the read-back of its
 * status word on the handle's stream, and returns. The next call plans while this
 * batch runs on the GPU. A step whose device wait gave up is reported by the next
 * zxh_sync, or by the next call of any other entry point that uses the device
 * (each settles the work in flight first). zxh_state_view / zxh_stream users
 * order their own work after it (same stream) or call zxh_sync. zxh_last_stats
 * reports the launches and passes of the last batch and 0 ms. No counterpart in
 * the reference. */
int zxh_apply_async(zxh_sim *sim, const zxh_gate *gates, size_t count);

/* Waits for the zxh_apply_async work in flight; ZXH_ERR_TIMEOUT if a step's device
 * wait gave up. ZXH_OK at once when nothing is in flight. */
int zxh_sync(zxh_sim *sim);

/* Replaces ZXH::measure (zxh.cpp:555-559, measure_common.cpp:73-92): draws shots
 * outcomes with the reference GPU sampler's uniform stream
 * (src/zxh/src/measure/measure_cuda.cu:387-516,642-691) and keeps them on the
 * device until zxh_get_results. */
int zxh_measure(zxh_sim *sim, size_t shots);

/* Replaces ZXH::get_results (zxh.cpp:561-564): copies the first shots cached
 * outcomes to words, ceil(n/64) uint64 per shot, bit q = virtual qubit q
 * (measure_result_pack.h:24-44 layout). */
int zxh_get_results(zxh_sim *sim, uint64_t *words, size_t shots);

/* The distinct outcomes of the last zxh_measure and how often each was drawn,
 * counted on the device (the reference's sample_counts unpacks every shot on the
 * host into a std::map, bindings.cpp:36-54 / zxh.cpp:842-871). words[i] (same
 * layout as zxh_get_results) was drawn counts[i] times, i < *n_unique, in
 * increasing order of the state's real index (not sorted by word). A word
 * repeats only where the affine map is singular (a CX whose control equals its
 * target, which the reference also accepts: zxh.cpp:282-287). words NULL:
 * only *n_unique is set (a size query; the counting done for it is kept for the
 * next call). ZXH_ERR_LIMIT if capacity < *n_unique. No draw since the last
 * zxh_execute / zxh_apply: *n_unique = 0. */
int zxh_counts(zxh_sim *sim, uint64_t *words, uint64_t *counts, size_t capacity, size_t *n_unique);

/* Replaces ZXH::measured_count (zxh.cpp:566-569). */
int zxh_measured_count(const zxh_sim *sim, size_t *out);

/* Replaces ZXH::get_state (zxh.cpp:579-636). out is a HOST buffer of out_elems
 * complex values (2^n required) in the handle's dtype, interleaved re/im. */
int zxh_get_state(zxh_sim *sim, void *out, size_t out_elems, int order);

/* Same as zxh_get_state but writes into a DEVICE buffer of 2^n elements. */
int zxh_get_state_device(zxh_sim *sim, void *out_device, size_t out_elems, int order);

/* Replace ZXH::required_M / num_qubits (zxh.cpp:638-646). */
int zxh_required_M(const zxh_sim *sim, size_t *out);
int zxh_num_qubits(const zxh_sim *sim, size_t *out);

/* Device view of the real-address state after zxh_execute: data pointer, number
 * of real address bits m (2^m elements), bytes per element, global phase. Applies
 * the phases carried over by the last zxh_apply first (see zxh_apply); after a
 * later zxh_apply, call it again before reading the state. */
int zxh_state_view(zxh_sim *sim, void **data, size_t *m_bits, size_t *elem_bytes, double *global_phase_re,
                   double *global_phase_im);

/* The handle's CUDA stream (cudaStream_t), for callers that time or order work. */
int zxh_stream(zxh_sim *sim, void **stream);

/* Launch statistics of the last zxh_execute / zxh_apply / zxh_measure: number of
 * kernels launched, number of full read-modify-write passes over the state, and
 * the device time of those kernels in milliseconds (CUDA events recorded on the
 * handle's stream around the launches). Any pointer may be NULL. */
int zxh_last_stats(const zxh_sim *sim, uint64_t *kernels, uint64_t *passes, double *device_ms);

/* Multinomial sampler that allocates nothing, for callers that cannot call
 * cudaMalloc (a process whose device memory is reserved once up front, a
 * framework whose own allocator owns the device, or a latency path that must not
 * take the CUDA allocator's locks). It has no counterpart in the reference. It
 * draws shots outcomes
 * from the 2^m_bits-amplitude device state `state` (dtype ZXH_C64 or ZXH_C128,
 * interleaved re/im, real-address order) with the same uniform stream and the
 * same output order as zxh_measure after zxh_set_seed(seed), and writes the
 * real index of each shot to the caller's DEVICE buffer real_out (shots
 * uint64). Work is enqueued on `stream` (a cudaStream_t, NULL = default stream)
 * and the call returns once it is done.
 * Limits: m_bits <= 28 (ZXH_ERR_LIMIT otherwise, before any GPU work). Its
 * working memory is one 2.25 MiB file-scope device array that every GPU loading
 * the library holds until exit and that all calls on a device share: calls that
 * overlap on the GPU race and must be serialised by the caller. The first call on
 * a device resolves that array's address (cudaGetSymbolAddress) and keeps it for
 * the process; make that first call before any stream capture, and make no call
 * after a cudaDeviceReset. Errors are reported through zxh_last_error(NULL). */
int zxh_sample_noalloc(const void *state, int dtype, size_t m_bits, uint64_t seed, size_t shots, uint64_t *real_out,
                       void *stream);

/* ---- Expectation values and adjoint gradients (no counterpart in the
 * reference, which has no observables) ---------------------------------------- */

/* One Pauli term of an observable: kind ZXH_TERM_Z (coef * Z_q0),
 * ZXH_TERM_ZZ (coef * Z_q0 Z_q1) or ZXH_TERM_X (coef * X_q0). At most 256 terms. */
enum { ZXH_TERM_Z = 1, ZXH_TERM_ZZ = 2, ZXH_TERM_X = 3 };
typedef struct zxh_term {
    uint32_t kind;
    uint32_t q0;
    uint32_t q1;
    uint32_t reserved;
    double coef;
} zxh_term;

/* <psi|H|psi> of the state left by the last zxh_execute / zxh_apply, reduced in
 * FP64 on the device. */
int zxh_expectation(zxh_sim *sim, const zxh_term *terms, size_t nterms, double *value);

/* Runs the recorded gate list forward (like zxh_execute, saving a copy of the
 * state after every `checkpoint_every` parameterised gates, 0 = no checkpoints),
 * then one reverse sweep over the state and lambda = H|psi>, and writes
 * value = <H> and grads[i] = d<H>/d(theta of recorded gate i) for every recorded
 * gate (0 for gates without a parameter). Parameterised gates: RZ, P, CP, RX and
 * U3 records with lambda = phi = 0 (RY). grads holds the recorded gate count
 * (CRz records count as two: P then CP). The reverse sweep uncomputes with the
 * inverse gates; at each checkpoint the uncomputed state is replaced by the
 * saved forward state, which bounds the drift. The sweep holds 2^n amplitudes
 * per state (n <= 40). After the call the state is the forward output again. */
int zxh_adjoint_gradient(zxh_sim *sim, const zxh_term *terms, size_t nterms, size_t checkpoint_every, double *value,
                         double *grads, size_t ngrads);

/* Number of recorded gates (after CRz / Rx lowering). */
int zxh_gate_count(const zxh_sim *sim, size_t *out);

/* ---- Batched circuits (no counterpart in the reference, which runs one circuit
 * per ZXH object) ---------------------------------------------------------------- */

/* Many independent circuits, each with its own qubit count (6..34), gate records
 * and observable: circuit c has records gates[gate_offsets[c] .. gate_offsets[c+1])
 * and terms terms[term_offsets[c] .. term_offsets[c+1]]. Every circuit is compiled
 * once at creation (every qubit expanded, X/CX transported) into a chain of
 * passes: |0...0>, general strided passes with fused diagonal windows, lambda =
 * H psi with <H>, and the adjoint reverse passes. All states live in one device
 * arena. Errors of creation are reported by zxh_batch_last_error(NULL). */
typedef struct zxh_batch zxh_batch;
enum { ZXH_BATCH_SEQUENTIAL = 0, ZXH_BATCH_PERSISTENT = 1, ZXH_BATCH_GRAPH = 2 };
int zxh_batch_create(zxh_batch **out, size_t count, const uint32_t *nqubits, const size_t *gate_offsets,
                     const zxh_gate *gates, const size_t *term_offsets, const zxh_term *terms, int dtype, int device);
int zxh_batch_destroy(zxh_batch *batch);
const char *zxh_batch_last_error(const zxh_batch *batch);
/* offsets[count + 1]: circuit c's gradients are grads[offsets[c] .. offsets[c+1]),
 * one per recorded gate after lowering (CRz records count as two). */
int zxh_batch_gradient_offsets(const zxh_batch *batch, size_t *offsets);
/* Energies (count) and gradients of every circuit. mode ZXH_BATCH_SEQUENTIAL runs
 * every pass as its own launch, circuit after circuit; ZXH_BATCH_PERSISTENT runs
 * all of them in one persistent kernel that takes tasks from a queue (a task
 * waits, bounded, for the previous pass of its circuit); ZXH_BATCH_GRAPH replays
 * that launch from a CUDA graph captured on first use. */
int zxh_batch_run(zxh_batch *batch, int mode, double *energies, double *grads, size_t ngrads);
/* Knobs: grow_regs (1..4, gates with high deltas per general strided pass),
 * adj_regs (1..3, the same for the reverse passes), task_items (pass items per
 * task), task_elems (amplitudes per task of the element-wise passes); setting
 * one of these recompiles the batch. threads (64, 128 or 256): threads per CTA
 * of the persistent kernel, i.e. the warps that work on one task.
 * wait_limit_log2 (0..31, default 31): a persistent task waits at most
 * 2^wait_limit_log2 SM clocks for the previous pass of its circuit, then the run
 * ends early and zxh_batch_run returns ZXH_ERR_TIMEOUT; the handle stays usable
 * (the next run starts from scratch). Small values exist to test that path. */
int zxh_batch_set(zxh_batch *batch, const char *name, int value);
int zxh_batch_get(const zxh_batch *batch, const char *name, int *value);
/* Times the persistent launch (reps timed runs per setting after one warm-up)
 * and keeps the fastest: grow_regs in {2, 3, 4} x task_items in {32, 128, 512,
 * 2048} (task_elems = 1024 x task_items), then threads in {64, 128, 256}, then
 * adj_regs in {1, 2, 3}, each at the best setting so far. */
int zxh_batch_tune(zxh_batch *batch, int reps);
/* ops and tasks of the compiled batch, device ms of the last run, and the
 * algorithmic state bytes of one run (each pass reads and writes its states once:
 * init 1x, forward and lambda passes 2x, adjoint passes 4x the state). */
int zxh_batch_stats(const zxh_batch *batch, uint64_t *ops, uint64_t *tasks, double *device_ms, uint64_t *bytes);

/* Host-only dry run of execute(): lowers the records, runs calc_mem, the
 * reference's execute() schedule and the pass planner, and launches nothing
 * (no CUDA call is made). out[13]: [0] M, [1] final real bits, [2..9] passes
 * per kind (product, expand, tile, pair, diagonal, fast low-qubit, strided
 * high-qubit, general strided), [10] state passes (all but product and the
 * |0...0> init), [11] Walsh-sum window passes, [12] span passes. No
 * counterpart in the reference. */
int zxh_plan_stats(size_t n, int disable_x, int eager_expand_all, int dtype, const zxh_gate *gates, size_t count,
                   uint64_t *out);

/* Host circuit compiler: the reference's boundary scheduler
 * (src/zxh/zxhsim/circ_optimizer.py:218-420, optimize_circuit) over gate records.
 * Single-qubit gates merge per qubit until a two-qubit gate or a barrier needs
 * the qubit and are re-emitted as RZ (+ X), H or U3; a CX between two pending
 * exact H gates is emitted reversed with the H's kept pending. level 0 emits every
 * gate at once (identities dropped), level >= 1 schedules. The result equals the
 * input up to a global phase. out may be NULL (a size query: *out_count gives
 * the size); with capacity < *out_count the call returns ZXH_ERR_LIMIT. Accepts the record
 * types zxh_push_gates accepts. No GPU work. */
int zxh_optimize_gates(size_t n, int level, const zxh_gate *gates, size_t count, zxh_gate *out, size_t capacity,
                       size_t *out_count);

/* Pass-planner tuning (used by the autotuner): tile_bits_c64, tile_bits_c128,
 * contig_bits, max_gates (generic tile pass), fast_gates (gates per fast U3
 * pass), fast_fuse_quad, fast_contig_c64, fast_contig_c128, row_wide_c64,
 * row_wide_c128 (shape of the strided high-qubit pass), diag_chunk_bits (log2
 * tiles a warp of the diagonal pass walks in Gray-code order; -1 = automatic),
 * diag_row_bits_c64, diag_row_bits_c128 (log2 rows of its warp tile), grow (1:
 * U3 batches whose pair deltas span several bits use the general strided pass,
 * 0: the TMA tile / global pair passes), grow_regs (1..4: gates with high deltas per
 * general strided pass), grow_only (1: plan every batch and window as general
 * strided passes after a |0...0> init, the pass set of the batched launch; needs
 * eager_expand_all), adj_windows (1: the adjoint sweep undoes diagonal gates
 * inside its general strided passes, 0: in separate diagonal-group passes),
 * adj_regs (1..4: gates with high deltas per reverse strided pass; 4 runs at one
 * CTA per SM), grow_staged (0..7, bit mask: general strided passes whose warps
 * stage their next item in shared memory with TMA bulk copies; 1 = the adjoint
 * sweep's in complex64, 2 = the forward ones, 4 = the adjoint sweep's in
 * complex128),
 * low_pass (1: gates on the lane / vector bits ride in a strided low pass with
 * lane bits swapped into registers, 0: the TMA fast tile pass), low_regs_c64,
 * low_regs_c128 (0..4: register-bit gates that join the low pass), real_split
 * (1: single-bit U3 gates run as real rotations with their phases in the
 * windows), diag_prefetch_c64, diag_prefetch_c128 (1: the diagonal pass stages
 * each warp's next tile with a TMA bulk copy), walsh (1: a window whose
 * selectors are parities of several real bits runs as one Walsh-sum pass, its
 * cost per amplitude independent of the window's size; 0: general terms
 * evaluated per amplitude, 32 per pass), walsh_min_general (general terms from
 * which a standalone window takes the Walsh pass; 0 = every one), span (1:
 * U3 batches run as span passes, the gates on the low 13 (complex64) or 12
 * (complex128) bits in one pass and up to 10 / 9 high-bit gates per pass; 0: the
 * register-row passes), span_min_run (3..8: log2 of the shortest contiguous run
 * a strided span pass reads), span_land (1: the span pass's next tile lands in
 * shared memory while the current one is worked on; 0: tiles loaded straight
 * into registers), span_split (0: the high-bit gates dealt to the strided span
 * passes in blocks of neighbouring bits, the larger blocks on the lower bits; 1:
 * round robin; 2: blocks, the larger on the higher bits), span_order (0: the
 * strided span passes from the lowest bits up, but the first one that runs two
 * layouts moved to the front, so the window before the batch rides on it; 1:
 * from the lowest bits up; 2: from the highest down), span_mixed (1: a U3 batch
 * mixing gates with single-bit pair deltas (at least 8) and gates whose deltas
 * span several bits runs the single-bit ones as span passes first and the rest
 * as general strided passes; 0: all as general strided passes). Takes effect at
 * the next zxh_execute / zxh_apply. No
 * counterpart in the reference. */
int zxh_set_param(zxh_sim *sim, const char *name, int value);

#ifdef __cplusplus
}
#endif

#endif /* ZXH_B200_H */
