/*
 * pq_oracle.h -- TEST INFRASTRUCTURE, not product code.
 *
 * C ABI of the CPU oracle: a plain C++17 restatement of propaq's numerical
 * propagation engine (hkbelagali/propaq, crates/core/src/engine/termsum.rs,
 * crates/core/src/engine/partitioned_termsum.rs, crates/pauli/src/engine.rs,
 * crates/majorana/src/engine.rs).  It is the checker the CUDA engine is compared
 * against, and the timed CPU baseline.  Only tests/, __graft_entry__.smoke() and
 * bench.py (its cpu_baseline / reference arm) load it.
 */
#ifndef PQ_ORACLE_H
#define PQ_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Noise resolution kinds (crates/core/src/engine/noise_resolver.rs:28-37). */
enum {
  PQO_NOISE_NONE = 0,
  PQO_NOISE_TABLE = 1,   /* one weight table, n_units + 1 entries            */
  PQO_NOISE_LAYERED = 2, /* one weight table per circuit layer (caller-built) */
  PQO_NOISE_PLUGIN = 3,  /* a loaded native noise plugin, resolved by depends */
};

typedef struct pqo_config {
  uint32_t basis_kind;    /* 0 = Pauli, 1 = Majorana                          */
  uint32_t n_units;       /* qubits (Pauli) or sites = modes / 2 (Majorana)   */
  uint32_t n_words;       /* u64 words per key (dispatch width W)             */
  uint32_t n_partitions;  /* hash partitions = worker threads (>= 1)          */
  int64_t max_weight;     /* < 0: no WeightTruncator                          */
  uint32_t has_min_coeff; /* CoefficientTruncator present                     */
  double min_coeff;
  int64_t min_terms;      /* < 0: no TermBudget                               */
  void* truncator;        /* pqo_plugin* from pqo_load_truncator, or NULL     */
  uint32_t noise_kind;    /* PQO_NOISE_*                                      */
  const double* noise_tables; /* TABLE: table_len; LAYERED: n_layers*table_len */
  size_t noise_table_len;
  void* noise_plugin;     /* pqo_plugin* from pqo_load_noise (PLUGIN kind)    */
} pqo_config;

typedef struct pqo_result {
  double expectation;          /* per-partition row-order sums, then summed  */
  double expectation_accurate; /* compensated (Neumaier) sum of all terms     */
  double expectation_abs;      /* sum of |c * trace|: the sum's condition     */
  uint64_t terms_below_cutoff;
  uint64_t n_final;            /* live terms at the end                       */
  uint64_t emitted, hits, visited, declined;
  double discarded_l1;
} pqo_result;

/* Loads a plugin with the reference loader's validation
 * (crates/core/src/policy/native_noise.rs:217-288,
 *  crates/core/src/policy/native_truncator.rs:205-276).
 * Returns 0 on success; 1 = load failure (OSError), 2 = validation (ValueError).
 * On error `err` receives the message. */
int pqo_load_noise(const char* path, const char* config_json, void** out, char* err, size_t err_len);
int pqo_load_truncator(const char* path, const char* config_json, void** out, char* err, size_t err_len);
void pqo_plugin_free(void* plugin);
uint32_t pqo_plugin_depends(const void* plugin);

/* Runs the engine.  Gates are in Heisenberg application order (circuit layers
 * reversed, gates within each layer reversed, as extract_layers does,
 * crates/pauli/src/engine.rs:44-70); layer l covers gates
 * [layer_offsets[l], layer_offsets[l+1]).  diag_state may be NULL (no
 * expectation).  n_terms_out receives the live count after each gate.
 * Returns an opaque handle holding the final terms (NULL on error; see
 * pqo_last_error). */
void* pqo_run(const pqo_config* cfg, const uint64_t* obs_words, const double* obs_coeffs,
              size_t n_obs, const uint64_t* gate_words, const double* gate_angles,
              size_t n_gates, const uint32_t* layer_offsets, size_t n_layers,
              const uint64_t* diag_state, size_t diag_words, uint64_t* n_terms_out,
              pqo_result* out);
/* Final terms with the deferred Clifford frame applied and its sign folded
 * into the coefficient (crates/pauli/src/engine.rs:216-224). */
size_t pqo_terms_count(const void* run);
void pqo_terms_copy(const void* run, uint64_t* keys, double* coeffs);
void pqo_run_free(void* run);
const char* pqo_last_error(void);

/* Algebra probes for unit tests (one key at a time). */
uint32_t pqo_weight(uint32_t basis_kind, uint32_t n_units, uint32_t n_words, const uint64_t* key);
int pqo_anticommutes(uint32_t basis_kind, uint32_t n_words, const uint64_t* gen, const uint64_t* key);
/* product G*key -> child words, returns the phase exponent p (phase = i^p). */
int pqo_product(uint32_t basis_kind, uint32_t n_words, const uint64_t* gen, const uint64_t* key,
                uint64_t* child);
double pqo_trace(uint32_t basis_kind, uint32_t n_units, uint32_t n_words, const uint64_t* key,
                 const uint64_t* diag_state, size_t diag_words);

#ifdef __cplusplus
}
#endif
#endif
