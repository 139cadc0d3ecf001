/*
 * propaq_cuda.h -- C ABI of the B200 propagation engine (libpropaq_cuda.so).
 *
 * The engine applies a circuit of Pauli/Majorana rotations to a sparse sum of
 * packed bitstrings with FP64 coefficients in the Heisenberg picture: it
 * branches anticommuting terms, merges duplicates, truncates by weight and
 * coefficient, damps by noise, and reduces the expectation value against a
 * computational-basis state.  Everything between the first and last call of
 * pq_run happens on one GPU.
 *
 * Every entry point below replaces one interface of the reference
 * (hkbelagali/propaq); each comment names the file:line it stands in for.
 *
 * Conventions
 *   - Keys are `n_words` u64 words per term, two bits per unit, interleaved:
 *     Pauli qubit q uses bit 2q (x) and 2q+1 (z); Majorana mode m uses bit m,
 *     so site k owns modes 2k and 2k+1 (crates/pauli/src/algebra.rs:242-257,
 *     crates/majorana/src/algebra.rs:218-233).  n_words comes from
 *     pq_words_for_units (crates/pauli/src/engine.rs:289-301).
 *   - All functions return PQ_OK (0) or a PQ_ERR_* code; no exception crosses
 *     the ABI.  pq_engine_last_error gives the message of the last failure.
 *   - The engine owns all device memory; the caller owns every host array.
 *     One engine = one CUDA stream; an engine is not re-entrant, distinct
 *     engines may be used from distinct threads.
 */
#ifndef PROPAQ_CUDA_H
#define PROPAQ_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PQ_ABI_VERSION 1u

/* Status codes.  The Python layer maps them to the reference's exception
 * types: INVALID -> ValueError (crates/pauli/src/propagator.rs:256-260),
 * CEILING -> RuntimeError (crates/core/src/storage/operator_index.rs:116-127),
 * PLUGIN_LOAD -> OSError and PLUGIN -> ValueError
 * (crates/core/src/policy/native_noise.rs:217-260). */
enum {
  PQ_OK = 0,
  PQ_ERR_INVALID = 1,        /* bad argument, width beyond 2048 units, odd modes */
  PQ_ERR_CUDA = 2,           /* CUDA runtime failure or no usable device          */
  PQ_ERR_OOM = 3,            /* device allocation failed                          */
  PQ_ERR_CEILING = 4,        /* live terms would exceed the engine's row ceiling  */
  PQ_ERR_PLUGIN_LOAD = 5,    /* dlopen failed                                     */
  PQ_ERR_PLUGIN = 6,         /* plugin symbol / ABI / dependency validation       */
  PQ_ERR_DEVICE_TIMEOUT = 7, /* a bounded device-side wait expired                */
  PQ_ERR_UNSUPPORTED = 8     /* a configuration this build does not run           */
};

enum { PQ_BASIS_PAULI = 0, PQ_BASIS_MAJORANA = 1 };

/* How noise reaches the engine (crates/core/src/engine/noise_resolver.rs:28-37). */
enum {
  PQ_NOISE_NONE = 0,
  PQ_NOISE_TABLE = 1,   /* one factor per weight, table_len entries              */
  PQ_NOISE_LAYERED = 2, /* n_layers tables of table_len entries, one per layer   */
  PQ_NOISE_PLUGIN = 3   /* a loaded plugin; the engine resolves it by `depends`  */
};

typedef struct pq_engine pq_engine;
typedef struct pq_plugin pq_plugin;

/* One run's truncation and noise, the flattened form of
 * crates/core/src/policy/truncators.rs:188-213 (ResolvedConfig) plus the
 * resolved noise model. */
typedef struct pq_run_config {
  uint32_t basis_kind;       /* PQ_BASIS_*                                      */
  uint32_t n_units;          /* qubits (Pauli) or sites = modes / 2 (Majorana)  */
  int64_t max_weight;        /* WeightTruncator; < 0 = none                     */
  uint32_t has_min_coeff;    /* CoefficientTruncator present                    */
  double min_coeff;
  int64_t min_terms;         /* TermBudget floor; < 0 = none                    */
  const pq_plugin* truncator;/* NativeTruncator, or NULL                        */
  uint32_t noise_kind;       /* PQ_NOISE_*                                      */
  const double* noise_tables;/* TABLE / LAYERED factors                         */
  size_t noise_table_len;    /* entries per table (normally n_units + 1)       */
  const pq_plugin* noise_plugin; /* PLUGIN kind                                 */
  uint32_t want_terms;       /* keep the final terms for pq_result_terms: 1 in
                                the engine's row order, 2 sorted by key (as a
                                64 n_words-bit integer, on the device)          */
  uint32_t blocks_per_sm;    /* sweep blocks per SM; 0 = by live count: 1 while
                                every row has a thread, 2 up to 2^20 rows, then
                                as many as fit (a launch stops and is relaunched
                                when its live count outgrows its grid)          */
  uint32_t log_gates;        /* keep per-gate records for pq_result_gates (the
                                Logger's verbose log); rotations then run one op
                                each, unfused, so each has its own device time  */
  /* Tuning; 0 = the engine's default.  Results do not depend on them. */
  uint32_t fuse_max;         /* consecutive commuting rotations run in one pass
                                over the rows: 1-2 (default 2)                  */
  uint32_t tile_items;       /* rows per thread of a many-row gate tile: 1-4
                                (default 4)                                     */
  uint32_t bucket_slots;     /* hash-table slots a key's probe starts in: 2, 4
                                or 8 (default 2)                                */
} pq_run_config;

/* crates/core/src/interface/results.rs:8-51 (PropagationResult), plus the
 * engine's own counters. */
typedef struct pq_result {
  double expectation_value;   /* 0 when no diag_state was given               */
  uint64_t terms_below_cutoff;/* live terms with |c| < min_coeff at the end   */
  uint64_t sparse_key_bytes;  /* device bytes holding keys and the hash table */
  uint64_t n_final;           /* live terms at the end                        */
  uint64_t n_layers_run, n_gates_run;
  uint64_t gpu_launches;      /* kernels this run launched                    */
  uint64_t peak_terms;        /* largest live count seen                      */
  double device_ms;           /* device time from the first sweep launch to the
                                 expectation value (CUDA events, engine stream) */
  double sweep_ms;            /* CUDA-event time of the sweep kernel launches  */
  uint64_t sweep_launches;    /* 1, plus one per capacity growth               */
  /* Split of the sweep time by op kind, from the device clock at each op's end. */
  double gate_ms, noise_ms, phase_ms;
  uint64_t gate_ops, noise_ops, phase_ops;
  uint64_t sum_rows_gate;     /* sum over gate ops of the live rows they scan  */
  uint64_t sum_anti;          /* ... of the rows anticommuting with the gate   */
  uint64_t sum_children;      /* ... of the children they append               */
  uint64_t sum_rows_phase;    /* sum over phase-only ops of the rows they scan */
  uint64_t sum_rows_noise;    /* sum over noise ops of the rows they scan      */
  uint64_t sum_kept;          /* ... of the rows a reclaim keeps               */
  uint64_t class_ops;         /* ops that ran a class of rotations (generators on
                                 disjoint units) through one pass              */
} pq_result;

/* Key width for a register: 1,2,4,...,64 words for up to 32,64,...,2048
 * qubits (Pauli) or sites (Majorana); 0 if beyond the 2048-unit maximum.
 * Replaces runner_for, crates/pauli/src/engine.rs:289-301. */
uint32_t pq_words_for_units(uint32_t n_units);

/* Creates an engine on CUDA device `device`.  Replaces the rayon pool of
 * crates/core/src/engine/run_config.rs:13-55. */
int pq_engine_create(pq_engine** out, int device);
void pq_engine_destroy(pq_engine* engine);
const char* pq_engine_last_error(const pq_engine* engine);

/* Limits of one engine; a zero field keeps its default.  The reference's
 * counterparts are fixed: its term index ceiling
 * (crates/core/src/storage/operator_index.rs:116-127, TermIndexCeilingReached
 * -> RuntimeError) and the host's allocator.  Here a caller may lower the
 * ceiling and give the engine a device-memory budget; a run that needs more
 * fails with PQ_ERR_CEILING / PQ_ERR_OOM and the engine stays usable.  The
 * wait limits bound the device's grid barrier and look-back spins (a wait
 * that runs out ends the launch with PQ_ERR_DEVICE_TIMEOUT instead of
 * hanging); hold_block / hold_us exist for tests of that path: one block of
 * every sweep launch waits hold_us microseconds (at most 100 ms) before its
 * first op, so that short wait limits run out. */
typedef struct pq_engine_limits {
  uint64_t max_rows;         /* live-term ceiling (rounded down to a power of two);
                                0 = 2^31, the table's row index                 */
  uint64_t max_device_bytes; /* device memory the engine's buffers may hold; 0 = any */
  uint32_t barrier_spins;    /* polls of a grid-barrier wait; 0 = 2^25 (~2 s)   */
  uint32_t lookback_spins;   /* polls of a tile look-back wait; 0 = 2^22 (~0.3 s) */
  uint32_t hold_block;       /* block (of a launch, or of a batch instance's slice) */
  uint32_t hold_us;          /* that waits before its first op; 0 = none        */
} pq_engine_limits;
/* NULL restores every default.  Applies to the engine's later runs. */
int pq_engine_set_limits(pq_engine* engine, const pq_engine_limits* limits);
/* Device bytes the engine holds in buffers allocated since its limits were
 * last set (what max_device_bytes is compared with). */
uint64_t pq_engine_device_bytes(const pq_engine* engine);

/* Runs one propagation; replaces engine::run / run_at_width
 * (crates/pauli/src/engine.rs:74-238, :305-357; crates/majorana/src/engine.rs).
 *
 *   obs_words   n_obs * n_words   observable keys (duplicates are added)
 *   obs_coeffs  n_obs             observable coefficients
 *   gate_words  n_gates * n_words generators in HEISENBERG order: circuit
 *                                 layers reversed and the gates of each layer
 *                                 reversed (extract_layers, engine.rs:44-70)
 *   gate_angles n_gates           rotation angles (U = exp(-i angle G / 2))
 *   layer_offsets n_layers + 1    layer l holds gates [off[l], off[l+1])
 *   diag_state  diag_words        computational-basis state, one bit per unit;
 *                                 NULL = no expectation value
 *   n_terms_out n_gates           live terms after each gate (may be NULL)
 */
int pq_run(pq_engine* engine, const pq_run_config* cfg, const uint64_t* obs_words,
           const double* obs_coeffs, size_t n_obs, const uint64_t* gate_words,
           const double* gate_angles, size_t n_gates, const uint32_t* layer_offsets,
           size_t n_layers, const uint64_t* diag_state, size_t diag_words,
           uint64_t* n_terms_out, pq_result* out);

/* Final terms of the last run with want_terms, with the deferred Clifford
 * frame applied and its sign folded into the coefficient
 * (crates/pauli/src/engine.rs:216-224, partitioned_termsum.rs:265-272).
 * Writes min(cap, n) terms, returns n. */
size_t pq_result_terms(pq_engine* engine, uint64_t* keys, double* coeffs, size_t cap);

/* One gate's record of the last pq_run made with log_gates: the reference's
 * GateRecord (crates/pauli/src/engine.rs:252-265, written to the verbose log
 * by crates/pauli/src/propagator.rs:23-73) with the device's time. */
typedef struct pq_gate_record {
  uint64_t terms_before, terms_after; /* live terms around the gate             */
  uint64_t terms_gained;              /* rows the gate created                  */
  uint64_t declined;                  /* sin branches the emit check held back  */
  uint64_t emitted;                   /* sin branches that went out             */
  uint64_t exchange_hits;             /* ... onto a row that was already live   */
  double discarded_coeff_l1;          /* sum of |held branch| that no partner
                                         claimed (termsum.rs:604-628)          */
  double discarded_coeff_max;         /* largest of those                       */
  double elapsed_ms;                  /* device time of the gate's op; 0 for a
                                         rotation deferred into the Clifford frame */
  uint32_t layer_idx;                 /* layer in Heisenberg order              */
  int32_t op;                         /* the gate's op in the sweep; -1 = deferred */
} pq_gate_record;

/* Per-gate records of the last pq_run, gates in Heisenberg order: live
 * counts and device time after every run (a fused op's time goes to its first
 * rotation), the emit statistics (declined, emitted, exchange_hits, the
 * discarded mass) only after a run made with log_gates.  Writes min(cap, n)
 * records, returns n. */
size_t pq_result_gates(pq_engine* engine, pq_gate_record* out, size_t cap);

/* One propagation of a batch: the arguments of pq_run in one record.  Keys
 * are pq_words_for_units(cfg.n_units) words wide. */
typedef struct pq_instance {
  pq_run_config cfg;
  const uint64_t* obs_words;
  const double* obs_coeffs;
  size_t n_obs;
  const uint64_t* gate_words;
  const double* gate_angles;
  size_t n_gates;
  const uint32_t* layer_offsets;
  size_t n_layers;
  const uint64_t* diag_state;
  size_t diag_words;
  uint64_t* n_terms_out;
  pq_result* result;
} pq_instance;

/* Grid sharing of pq_run_batch. */
typedef struct pq_batch_tuning {
  uint32_t blocks_per_sm;  /* grid size per SM; 0 = as many as fit              */
  uint32_t split;          /* 0: blocks shared equally among the instances;
                              1: in proportion to remaining ops x live terms    */
  uint32_t rebalance_pct;  /* when this % of the grid has been left by finished
                              instances, the others stop at their next op and
                              the grid is re-split among them; 0 = never        */
  uint32_t fuse_max;       /* as pq_run_config, for every instance; 0 = each
                              instance's own                                    */
  uint32_t tile_items;
  uint32_t bucket_slots;
} pq_batch_tuning;

/* Runs n independent propagations of one basis in shared persistent
 * launches: each instance owns a slice of the co-resident grid and runs its
 * op sequence there with its own grid barrier, so small instances fill the
 * GPU together and no instance pays a launch per gate.  The reference runs
 * such sweeps as one expectation_value call after another
 * (ZeroNoiseExtrapolator.run / ZeroCutoffExtrapolator.run,
 * propaq/extrapolators/zne.py:63-108, zce.py:88-137); each instance gives
 * pq_run's terms, coefficients and live counts on the same arguments (new rows
 * may be appended in another order, so the expectation sum agrees to its last
 * bits).
 *
 * Keys up to 2x narrower than the widest instance run at half its width;
 * narrower ones are widened with zero words (results are unchanged).
 * device_ms / sweep_ms of every result are the batch's.  A TermBudget floor
 * together with a weight cut and a weight-changing Clifford rotation needs the
 * live count on the host mid-run and is refused (PQ_ERR_UNSUPPORTED): run
 * that instance with pq_run.  tuning NULL = {0, 1, 25}. */
int pq_run_batch(pq_engine* engine, const pq_instance* instances, size_t n, const pq_batch_tuning* tuning);

/* Expectation value and its gradient with respect to every gate angle,
 * grad[g] = dE / d gate_angles[g], by reverse-mode differentiation of the
 * propagation with its truncation decisions (dropped, held and emitted
 * branches; reclaimed rows) held as the forward run made them.  This entry
 * point has no counterpart in the reference, whose only derivative-free
 * parameter sweep is surrogate evaluation (crates/surrogate/src/model.rs:63-107);
 * it backs a torch.autograd.Function over the propagators.
 *
 * Arguments as pq_run; diag_state is required.  The forward run records what
 * the reverse pass needs into a pool of record_bytes of device memory: 12
 * bytes per row entering each rotation.  0 = the size the engine's last
 * default-sized gradient needed plus a quarter (at first 40% of the free
 * memory, at most 48 GB); the engine keeps the pool, the adjoint vectors and
 * the checkpoints between calls and frees them in pq_engine_destroy.  When it
 * all fits, one reverse sweep follows.  Otherwise the
 * forward run's terms at the start of every checkpoint_layers layers (0 = one
 * segment) are used to re-run one segment at a time while recording.  Gates
 * deferred into the Clifford frame (fixed Clifford rotations) get NaN.  A
 * TermBudget floor with a weight cut and a weight-changing Clifford rotation
 * is refused (PQ_ERR_UNSUPPORTED), as are truncator plugins and key-reading
 * noise.  out->device_ms covers both passes. */
int pq_run_adjoint(pq_engine* engine, const pq_run_config* cfg, const uint64_t* obs_words,
                   const double* obs_coeffs, size_t n_obs, const uint64_t* gate_words,
                   const double* gate_angles, size_t n_gates, const uint32_t* layer_offsets,
                   size_t n_layers, const uint64_t* diag_state, size_t diag_words,
                   uint32_t checkpoint_layers, uint64_t record_bytes, double* grad,
                   uint64_t* n_terms_out, pq_result* out);

/* Final terms of instance `index` of the last batch (index 0 after pq_run),
 * as pq_result_terms. */
size_t pq_result_terms_at(pq_engine* engine, size_t index, uint64_t* keys, double* coeffs, size_t cap);

/* Plugins: the reference's loader and validation, byte for byte the same
 * symbol names (crates/core/src/policy/native_noise.rs:217-288,
 * crates/core/src/policy/native_truncator.rs:205-276). */
int pq_plugin_load_noise(const char* path, const char* config_json, pq_plugin** out,
                         char* err, size_t err_len);
int pq_plugin_load_truncator(const char* path, const char* config_json, pq_plugin** out,
                             char* err, size_t err_len);
void pq_plugin_free(pq_plugin* plugin);
/* A noise model given as a function of the caller's, with the plugin ABI's
 * factor signature; `depends` as propaq_noise_depends (bit 0 KEY, bit 1
 * LAYER).  It replaces the Python damping_factor_term hook path
 * (crates/core/src/engine/noise_resolver.rs:28-37, ResolvedNoise::PythonTerm;
 * crates/pauli/src/engine.rs:142-158): the host calls it for every live term
 * at each noise op.  Free with pq_plugin_free. */
typedef double (*pq_noise_factor_fn)(void* ctx, uint32_t basis_kind, const uint64_t* words, size_t n_words,
                                     uint32_t n_units, uint32_t weight, uint32_t layer_index,
                                     uint32_t n_layers);
int pq_plugin_from_callback(pq_noise_factor_fn fn, void* ctx, uint32_t depends, pq_plugin** out);
uint32_t pq_plugin_depends(const pq_plugin* plugin);
/* NativeNoiseModel.factor_term (native_noise.rs:316-333). */
double pq_plugin_noise_factor(const pq_plugin* plugin, uint32_t basis_kind, const uint64_t* words,
                              size_t n_words, uint32_t n_units, uint32_t weight,
                              uint32_t layer_index, uint32_t n_layers);
/* NativeTruncator.keep_term (native_truncator.rs:305-328); 1 = keep. */
int pq_plugin_truncator_keep(const pq_plugin* plugin, uint32_t basis_kind, const uint64_t* words,
                             size_t n_words, uint32_t n_units, uint32_t weight,
                             double coeff_magnitude, uint32_t layer_index, uint32_t n_layers);

/* Expectation value sum_i c_i <s|K_i|s> of a term sum held in HOST memory,
 * for callers that may not allocate device memory.  This entry point has no
 * counterpart in the reference.
 *
 * Who needs it: programs that own all device memory themselves -- frameworks
 * that reserve (almost) the whole GPU up front for their own allocators, or
 * applications with a fixed device-memory budget -- where a cudaMalloc from
 * inside the library fails or breaks the owner's accounting.  It allocates
 * nothing: the terms are staged into a static __device__ array of
 * PQ_NOALLOC_SCRATCH_BYTES, which every GPU that loads it holds until the
 * process exits.  n_terms * (8 * n_words + 8) bytes (plus 8.25 KiB of partial
 * sums) must fit; larger inputs are refused with PQ_ERR_INVALID and a message
 * in `err`.  n_units <= 256.
 *
 * Every call looks the array's address up in the current context (a
 * cudaGetSymbolAddress, which allocates nothing), so it stays right after a
 * cudaDeviceReset and in a context the caller created.  The array is
 * committed when the library's module is loaded on a device: at the first
 * call there (at library load under CUDA_MODULE_LOADING=EAGER, on every
 * device).  Make that first call before the program reserves its device
 * memory, and before any stream capture.  Every call shares the array, which
 * keeps the last call's contents: calls that overlap on one device race, so
 * serialise them.  n_terms = 0 gives 0.  Runs on the legacy default stream
 * and returns when the value has been copied to *out_value. */
#define PQ_NOALLOC_SCRATCH_BYTES (16u << 20)
int pq_expectation_noalloc(uint32_t basis_kind, uint32_t n_units, const uint64_t* keys,
                           const double* coeffs, size_t n_terms, const uint64_t* diag_state,
                           size_t diag_words, double* out_value, char* err, size_t err_len);

#ifdef __cplusplus
}
#endif
#endif /* PROPAQ_CUDA_H */
