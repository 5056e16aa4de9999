/*
 * mpx.h -- C ABI of the B200 propagation engine (libmpx.so).
 *
 * Plain C types only. Caller-owned host buffers are borrowed for the duration of a call; the device
 * term store is owned by the handle. One CUDA stream per handle; a handle is not thread-safe. Every
 * entry point returns an mpx_status; mpx_last_error() gives the message of the handle's last failure
 * (or of the last failed mpx_create on this thread when the handle is NULL).
 *
 * Each entry point replaces one method of the reference's per-tier engine class, reached from Python
 * through its nanobind module (src/monoprop/bindings/binder.h) and implemented in C++ by
 * MonomialPropagator<NumModes> (cpp/include/monoprop/MonomialPropagator.h); citations are to those files.
 *
 * Key layout (identical to the reference's, so keys compare word for word): a monomial over a storage
 * tier of T = ceil(num_modes/32)*32 modes is 2T bits in W = T/32 little-endian uint64 words, slot s at
 * bit 2T-1-s (cpp/monoprop/algebra/AlgebraCommon.h:45-52).
 */
#ifndef MPX_H
#define MPX_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MPX_API __attribute__((visibility("default")))
#else
#define MPX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MPX_OK = 0,
    MPX_ERR_INVALID = 1,  /* bad argument: reference raises ValueError / std::invalid_argument */
    MPX_ERR_CUDA = 2,     /* CUDA runtime error (message carries cudaGetErrorString) */
    MPX_ERR_NOMEM = 3,    /* device allocation failed */
    MPX_ERR_CAPACITY = 4, /* a bounded resource (fixed arena) is too small for the request */
    MPX_ERR_STATE = 5,    /* call not valid in the engine's current state: RuntimeError */
    MPX_ERR_NO_DEVICE = 6 /* no CUDA device / the sm_100a kernels cannot run here */
} mpx_status;

typedef enum { MPX_BASIS_MAJORANA = 0, MPX_BASIS_PAULI = 1 } mpx_basis;
typedef enum { MPX_CUTOFF_LENGTH = 0, MPX_CUTOFF_SUPPORT = 1 } mpx_cutoff_type;

typedef struct {
    int32_t basis;       /* mpx_basis; reference ctor kwarg basis= (binder.h:61-101) */
    int32_t cutoff_type; /* mpx_cutoff_type; kwarg cutoff_type= */
    uint32_t cutoff;     /* kwarg cutoff= */
    int32_t has_lower_atol;
    double lower_atol; /* kwarg lower_atol= (valid iff has_lower_atol) */
    int32_t has_upper_atol;
    double upper_atol;     /* kwarg upper_atol= (valid iff has_upper_atol) */
    int32_t num_modes;     /* logical modes (qubits in the Pauli basis); kwarg logical_num_modes= */
    int32_t device;        /* CUDA device ordinal */
    uint64_t capacity_hint; /* initial term capacity; 0 = automatic. The store grows on demand. */
    int32_t blocks_per_sm;  /* tuning: per-gate kernel grid, blocks per SM (1..4); 0 = 4 */
    int32_t table_shift;    /* tuning: hash table slots = next_pow2(capacity << table_shift) (1..3): load
                               factor <= 1/2, 1/4, 1/8; 0 = 1 */
    /* Schrodinger picture (kwarg schrodinger_cutoff=, MonomialPropagator.inl:146-179): when
     * has_schrodinger, the store starts as every fully paired monomial of at most
     * ceil(min(schrodinger_cutoff, 2 * logical modes) / 2) mode pairs over the logical modes, each holding its
     * reference-state score (generate_paired_op, MajoranaAlgebra.h:127-160); the observable is kept apart,
     * gates run first to last at the negated angle, an appended partner starts from its score
     * (FusedApply.h:39-83), and <O> = core + observable . state (MPFunctions.cpp:196-205). Graphs replay
     * from the dense reference state (every stored term at its score), the adjoint starts from the
     * observable, paring keeps the observable's terms above the threshold, and gradients are returned per
     * circuit layer as in the Heisenberg picture. */
    int32_t has_schrodinger;
    int32_t schrodinger_cutoff;
    int32_t logical_num_modes; /* modes the paired initial state spans (0 = num_modes) */
} mpx_config;

typedef struct mpx_engine mpx_engine;

/* Construct the Heisenberg term store from an encoded observable.
 * Replaces MonomialPropagator<N>::MonomialPropagator (MonomialPropagator.h:73-84; body
 * MonomialPropagator.inl:73-188). obs_words: [n_obs][W] distinct non-empty keys; obs_coef: encoded real
 * coefficients (Pauli: real part; Majorana: coeff / i^C(|M|,2)); core: the encoded empty-monomial
 * coefficient; state_mask: [W] key with slot 2m set for every occupied mode m of the reference state. */
MPX_API mpx_status mpx_create(const mpx_config *cfg,
                      const uint64_t *obs_words,
                      const double *obs_coef,
                      uint64_t n_obs,
                      double core,
                      const uint64_t *state_mask,
                      mpx_engine **out);

/* Heisenberg propagation: applies gen_words[n_layers-1] first down to gen_words[0], each rotation
 * exp(+i angle G) with angle = theta[mapping]*gen_coeff already mapped (MPFunctions.cpp:57-69).
 * Replaces MonomialPropagator<N>::propagate (MonomialPropagator.h:121-125, .inl:692-718).
 * gen_words: [n_layers][W]. Host buffers. */
MPX_API mpx_status mpx_propagate(mpx_engine *e, const uint64_t *gen_words, const double *angles, uint64_t n_layers);

/* A circuit uploaded once to device memory as per-gate descriptors, for repeated propagation (the
 * reference re-expands the circuit on every call: monomial_propagator.py:257-283). Angles can be
 * replaced without re-uploading the generators. */
typedef struct mpx_circuit mpx_circuit;
MPX_API mpx_status mpx_circuit_upload(mpx_engine *e, const uint64_t *gen_words, const double *angles, uint64_t n_layers,
                              mpx_circuit **out);
MPX_API mpx_status mpx_circuit_set_angles(mpx_engine *e, mpx_circuit *c, const double *angles);
MPX_API mpx_status mpx_propagate_circuit(mpx_engine *e, const mpx_circuit *c);
MPX_API void mpx_circuit_destroy(mpx_circuit *c);

/* <0|O|0> of the current operator: core + sum of phase*c over fully paired terms.
 * Replaces MonomialPropagator<N>::expectation_value with empty parameters (.inl:1034-1041,
 * MPFunctions.cpp:196-205). */
MPX_API mpx_status mpx_expectation(mpx_engine *e, double *out);

/* Number of terms in the store. Replaces MonomialPropagator<N>::size (MonomialPropagator.h:100). */
MPX_API mpx_status mpx_size(mpx_engine *e, uint64_t *out);

/* Words per key (W). */
MPX_API mpx_status mpx_words(mpx_engine *e, uint32_t *out);

/* Raw export of every stored key and its FP64 coefficient, in storage order, up to cap terms.
 * Replaces the raw read behind MonomialPropagator<N>::evolved_operator_terms (.inl:1099-1127) before its
 * atol filter, decoding and 1e-12 rounding (those stay on the host side). */
MPX_API mpx_status mpx_export(mpx_engine *e, uint64_t *words, double *coefs, uint64_t cap, uint64_t *n_out);

/* Per applied gate of the last propagate call, in application order: {n_g, a_g, e_g, m_g} =
 * terms before the gate, anticommuting terms, emitted sine branches, appended terms. */
MPX_API mpx_status mpx_gate_stats(mpx_engine *e, uint64_t *out4, uint64_t max_gates, uint64_t *n_out);

/* Restore the operator the engine was created with (keeps allocations). */
MPX_API mpx_status mpx_reset(mpx_engine *e);

/* Setters mirroring the reference properties (binder.h:154-185; MonomialPropagator.h:168-211). */
MPX_API mpx_status mpx_set_cutoff(mpx_engine *e, uint32_t cutoff);
/* cutoff_type property setter (binder.h:176-184, update_cutoff_type): mpx_cutoff_type; Pauli engines accept
 * only MPX_CUTOFF_SUPPORT (the reference's CutoffConfigError, a ValueError). */
MPX_API mpx_status mpx_set_cutoff_type(mpx_engine *e, int32_t cutoff_type);
MPX_API mpx_status mpx_set_lower_atol(mpx_engine *e, int32_t has_value, double value);
MPX_API mpx_status mpx_set_upper_atol(mpx_engine *e, int32_t has_value, double value);

/* only_rotate_len_k of the next propagate, gradient forward or graph build calls (the argument of
 * MonomialPropagator::propagate and ::build_graph, MonomialPropagator.inl:696-718, binder.h:102-110;
 * semantics Scan.h:146-157,376-391 and FusedApply.h:46-52): a term with more than k set slots takes no
 * part in a gate (neither cos-scaled nor emitted), and a partner outside that set receives its sine term
 * unscaled. A gradient or graph keeps the k it was recorded with. k <= 0 clears it; k > 2*num_modes is
 * rejected with the reference's message. */
MPX_API mpx_status mpx_set_only_rotate_len_k(mpx_engine *e, int64_t k);

/* basis_change of a Majorana engine (the constructor argument, MonomialPropagator.inl:82-131,460-495):
 * rows[s] (W words, encoded like a key) is the monomial slot s maps to; n_rows must be 2*num_modes. The
 * structural cutoff of every emitted partner P is then judged on XOR_{s in P} rows[s] (change_basis,
 * MajoranaAlgebra.h:179-189), the Jordan-Wigner image cutoff. n_rows = 0 clears it. Pauli engines reject
 * it with the reference's message. */
MPX_API mpx_status mpx_set_basis_change(mpx_engine *e, const uint64_t *rows, uint32_t n_rows);

/* Device pointers of the live store (keys [n][W], coefficients [n]) for in-process consumers such as
 * the torch wrapper; valid until the next mutating call. */
MPX_API mpx_status mpx_device_view(mpx_engine *e, const uint64_t **keys, double **coefs, uint64_t *n);

/* CUDA stream (cudaStream_t, as void*) the engine launches on. */
MPX_API mpx_status mpx_stream(mpx_engine *e, void **stream);

/* Number of engine kernel launches issued since the engine was created. */
MPX_API mpx_status mpx_launch_count(mpx_engine *e, uint64_t *out);

/* Number of propagations of a resident circuit (mpx_circuit_upload) whose streaming gate range ran as one
 * replayed CUDA graph. A range is captured after a propagation that did not grow the store (from the gate
 * where the shared-memory path handed over) and replayed while the store, its scratch and the truncation
 * settings are unchanged. No reference counterpart (the reference is host-only). */
MPX_API mpx_status mpx_graph_replay_count(mpx_engine *e, uint64_t *out);

/* Gradient of <0|O|0> with respect to every gate angle (reverse mode over the frozen truncation structure
 * of the forward pass). Replaces the reference's graph build + replayed gradient,
 * MonomialPropagator<N>::build_graph (MonomialPropagator.inl:620-690) followed by
 * expectation_value_and_gradient (MonomialPropagator.inl:1044-1050, MPFunctions.cpp:207-246).
 * mpx_adjoint_forward resets the store to the initial operator, propagates circuit c saving the
 * coefficient array every segment_gates gates (0 = one segment) and returns <0|O|0>; the engine then holds
 * the evolved operator. mpx_adjoint_backward replays each segment from its checkpoint and returns
 * grad_angles[l] = d<0|O|0>/d(angle_l) for every circuit layer l, angle_l = theta[map_l] * g_l (host
 * buffer of c's n_layers doubles). Peak extra memory: the checkpoints plus, for the largest segment,
 * 12 bytes per anticommuting term-gate pair and 25 bytes per emitted sine branch. Once an engine has run
 * one gradient forward pass it knows how many undo records the circuit needs; when they (12 bytes each,
 * plus 16 bytes per recorded pair) fit in free device memory with room to spare, the next forward pass
 * logs them all and mpx_adjoint_backward runs the reverse sweep alone, without replaying segments
 * (mpx_adjoint_logged reports which). The gradient is the same either way. */
MPX_API mpx_status mpx_adjoint_forward(mpx_engine *e, const mpx_circuit *c, uint64_t segment_gates, double *expectation);
MPX_API mpx_status mpx_adjoint_backward(mpx_engine *e, const mpx_circuit *c, double *grad_angles);
/* *out = 1 if the last mpx_adjoint_forward logged everything the reverse sweep needs, else 0. */
MPX_API mpx_status mpx_adjoint_logged(mpx_engine *e, int32_t *out);

/* Batch of independent problems (observable + circuit + angles each) on one GPU. No reference
 * counterpart: the reference runs one propagator per process (its benches loop over instances). Items
 * are spread over opt->workers host threads, each with its own engine and CUDA stream, deepest circuit
 * first, so the per-gate kernels of different instances share the GPU. An instance starts only while the
 * expected device footprints of the running ones (learned from the finished instances at least as deep)
 * fit the free memory measured at the start; one that still runs out of device memory waits for another
 * to finish and retries. Per item: <0|O|0> into *expectation, and with
 * opt->gradient d<0|O|0>/d(angle_l) into grad_angles[n_layers] (when non-NULL). */
typedef struct {
    const uint64_t *obs_words; /* [n_obs][W] */
    const double *obs_coef;
    uint64_t n_obs;
    double core;
    const uint64_t *state_mask; /* [W] */
    const uint64_t *gen_words;  /* [n_layers][W] */
    const double *angles;       /* [n_layers], theta[map] * g */
    uint64_t n_layers;
    double *expectation;  /* out */
    double *grad_angles;  /* out [n_layers], or NULL */
    uint64_t *final_terms; /* out (store size after propagation), or NULL */
    /* optional raw export of the evolved store, as mpx_export (NULL = none): up to export_cap keys
     * [export_cap][W] and coefficients in storage order; *export_n = the store size */
    uint64_t *export_words;
    double *export_coefs;
    uint64_t export_cap;
    uint64_t *export_n;
} mpx_batch_item;

typedef struct {
    int32_t workers;        /* instances in flight (0 = 8) */
    int32_t gradient;       /* also the adjoint gradient */
    uint64_t segment_gates; /* gradient checkpoint interval (0 = one segment) */
} mpx_batch_options;

MPX_API mpx_status mpx_batch_run(const mpx_config *cfg, mpx_batch_item *items, uint64_t n_items,
                                 const mpx_batch_options *opt, char *err, size_t err_len);

/* Frozen structure ("graph"), the reference's variational loop: MonomialPropagator<N>::build_graph
 * (MonomialPropagator.inl:620-690) keeps every truncation decision of a coefficient-informed build, and
 * expectation_value(parameters) / expectation_value_and_gradient(parameters) (.inl:1035-1050,
 * MPFunctions.cpp:196-246) replay it at new parameters. mpx_graph_build propagates circuit c at its current
 * angles (the engine then holds that evolved operator) and keeps each gate's rotated and appended pairs;
 * mpx_circuit_set_angles then changes the parameters and mpx_graph_expectation / mpx_graph_gradient
 * evaluate the frozen structure there (the engine then holds the replayed operator). grad_angles[l] =
 * d<0|O|0>/d(angle_l). Any other propagation of the engine keeps the graph; a rebuild replaces it. */
MPX_API mpx_status mpx_graph_build(mpx_engine *e, const mpx_circuit *c, uint64_t segment_gates, double *expectation);
MPX_API mpx_status mpx_graph_expectation(mpx_engine *e, const mpx_circuit *c, double *expectation);
MPX_API mpx_status mpx_graph_gradient(mpx_engine *e, const mpx_circuit *c, uint64_t segment_gates, double *expectation,
                                      double *grad_angles);

/* Pares the stored graph of circuit c against the reference state (the pare_threshold of the reference's
 * expectation_value[_and_gradient]_functional: pare_graph, PareGraph.cpp:103-141, keep set
 * indices_above(threshold), MonomialPropagator.inl:950-960). Terms whose reference-state weight exceeds
 * threshold are kept, and walking the layers backward so is every term whose value can still flow into a
 * kept one; later mpx_graph_expectation / mpx_graph_gradient calls skip the cos scaling of every other
 * term and the rotation of pairs with no kept endpoint. <0|O|0> and its gradient are unchanged for
 * threshold in [0, 1) (fully paired terms have weight 1); the replayed coefficients of pared terms are not
 * meaningful. threshold < 0 turns paring off. */
MPX_API mpx_status mpx_graph_pare(mpx_engine *e, const mpx_circuit *c, double threshold);

/* Pair log of a gradient forward pass (mpx_adjoint_forward, mpx_graph_build). The forward pass records
 * every gate's rotated and appended pairs (source, partner, phase), so that mpx_adjoint_backward replays
 * its segments without the hash resolve and mpx_graph_build needs no second pass; if the log overflows,
 * both replay the resolve instead (same results). capacity < 0: sized from the previous pass, at most half
 * the free device memory (default); 0: no log; > 0: that many records (9 bytes each). The reference's
 * graph build records the same pairs (MonomialPropagator.inl:620-690); this knob replaces nothing there. */
MPX_API mpx_status mpx_set_pair_log(mpx_engine *e, int64_t capacity);

/* Per-kernel timing. With profiling on, the sweep and resolve launches of every gate are bracketed by
 * CUDA events on the engine stream; mpx_kernel_times returns their summed device time (ms) for the last
 * propagate call. columns_ms is 0: no per-gate column launch remains (the resolve ORs the appended
 * terms' bit-columns). The reference has no device kernels; this replaces nothing there (its
 * closest counterpart is the per-layer wall time the bench harness records, benches/bench_models.py). */
MPX_API mpx_status mpx_set_profiling(mpx_engine *e, int32_t on);
MPX_API mpx_status mpx_kernel_times(mpx_engine *e, double *sweep_ms, double *resolve_ms, double *columns_ms,
                                    uint64_t *n_gates);

/* Device memory of all engines on a device comes from one library-owned pool that keeps freed memory
 * mapped for reuse, and freed blocks of 1 MiB or more are kept whole, per power-of-two size class, for
 * the next request of that class (so creating engines and regrowing stores does not re-map gigabytes
 * each time). This hands the kept blocks back to the pool and returns the pool's unused memory to the
 * driver. No reference counterpart (the reference is host-only). */
MPX_API mpx_status mpx_trim_device_memory(int32_t device);

/* Re-weights the initial operator. Replaces MonomialPropagator<N>::update_initial_operator (binder.h:153-156;
 * MonomialPropagator.h:277, MPOperator.h:193-232, Heisenberg branch): every key of words [n][W] must
 * already be in the store (the reference raises OperatorTermNotFound, a RuntimeError, otherwise: here
 * MPX_ERR_STATE with *missing = the index of the first absent key); the current coefficients become coefs
 * at those keys and zero elsewhere, and graph evaluations (mpx_graph_expectation / _gradient) start from
 * this operator until the next mpx_reset or mpx_graph_build. has_core: core replaces the empty-monomial
 * coefficient. */
MPX_API mpx_status mpx_update_initial_operator(mpx_engine *e, const uint64_t *words, const double *coefs, uint64_t n,
                                               int32_t has_core, double core, uint64_t *missing);

/* Device memory the engine holds, by part. Replaces the accounting behind the reference's
 * operator_memory_bytes / operator_memory_breakdown / graph_memory_bytes (binder.h:252-273,
 * MonomialPropagator.h:124-135): keys and coefficients at the store's capacity, the hash table, the
 * bit-column anticommutation index (the reference's InvertedIndex), per-gate scratch, the initial
 * operator, and the frozen graph (pairs and per-step arrays). */
typedef struct {
    uint64_t terms, capacity;
    uint32_t words;
    uint64_t key_bytes, coef_bytes, table_bytes, column_bytes, scratch_bytes, initial_bytes;
    uint64_t graph_layers, graph_pairs, graph_bytes;
} mpx_memory_info;
MPX_API mpx_status mpx_memory(mpx_engine *e, mpx_memory_info *out);

/* Frozen graph sizes. Replaces MonomialPropagator<N>::graph_size (MonomialPropagator.h:103-104):
 * *pairs = rotated and appended pairs over all layers (the reference's cycles), *cos_only = anticommuting
 * terms outside every pair (only cos-scaled), *layers = graph layers. All zero without a graph. */
MPX_API mpx_status mpx_graph_info(mpx_engine *e, uint64_t *layers, uint64_t *pairs, uint64_t *cos_only);

/* Deep copy of an engine: store, settings, re-weighted initial operator and frozen graph; with c (the
 * circuit of e's graph, or any circuit of e) also a copy of that circuit for the clone (*c_out). Replaces
 * the reference's __deepcopy__ (binder.h:113-116), which clones the operator store and shares the graph. */
MPX_API mpx_status mpx_clone(mpx_engine *e, const mpx_circuit *c, mpx_engine **out, mpx_circuit **c_out);

/* The calling thread's current CUDA device (the default device of new engines in the Python module). */
MPX_API mpx_status mpx_current_device(int32_t *device);

MPX_API const char *mpx_last_error(const mpx_engine *e);

/* <0|O|0> of a term store the caller holds in device memory, computed without allocating any device
 * memory. It has no counterpart in the reference (whose store never leaves the host); it is for callers
 * that cannot call cudaMalloc mid-run -- a host runtime that plans and owns all device memory and hands
 * this library pre-sized buffers, or one that cannot afford the device-wide synchronisation that
 * cudaMalloc/cudaFree imply. keys [n_terms][words] and coefs [n_terms] are device pointers in the layout
 * mpx_device_view exposes; state_mask is a HOST array of `words` words; out is a device pointer to one
 * double; stream is a cudaStream_t (NULL = legacy default stream); the call only enqueues work.
 * The scratch is a fixed 32 KiB array compiled into the library, so n_terms is limited to
 * 268435456 (larger stores return MPX_ERR_CAPACITY). The first call on each device does a one-time
 * set-up: it looks the array up with cudaGetSymbolAddress, so that device must be current, and that first
 * call should come before any stream capture on the device begins. Every call shares the one array: calls whose
 * kernels may overlap on the GPU must be serialised by the caller. The status covers this call's own
 * launches only (an error pending from the caller's earlier work is neither returned nor cleared); faults
 * during execution surface at the caller's next synchronisation. On failure a message is written to
 * err (up to err_len bytes, NUL-terminated) when err is not NULL. */
MPX_API mpx_status mpx_expectation_noalloc(int32_t basis, uint32_t words, const uint64_t *keys, const double *coefs,
                                           uint64_t n_terms, const uint64_t *state_mask, double core, double *out,
                                           void *stream, char *err, size_t err_len);
MPX_API void mpx_destroy(mpx_engine *e);

#ifdef __cplusplus
}
#endif

#endif /* MPX_H */
