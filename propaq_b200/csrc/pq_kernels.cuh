// pq_kernels.cuh -- kernel launch interface of the B200 propagation engine.
#pragma once

#include <cuda_runtime.h>

#include "pq_device.cuh"

namespace pq {

// One step of the op sequence a sweep runs.
enum OpKind : u32 {
  OP_GATE = 0,           // branch a rotation (pair rule, emit, append, insert)
  OP_PHASE = 1,          // |sin| < eps: scale the anticommuting rows by cos
  OP_NOISE_SCALE = 2,    // damp every row by its weight's factor
  OP_NOISE_COMPACT = 3,  // damp, then reclaim: filter + compact + re-insert
  OP_GATE2 = 4,          // this rotation and the next 1 / 2 / 3 (whose generators commute)
  OP_GATE_TAIL = 5,      // a later rotation of such a group: run by its head, skipped by the sweep
  OP_GATE3 = 6,
  OP_GATE4 = 7,
  // A class: the next m rotations (m in the bits above the low byte), whose
  // generators act on pairwise disjoint units, in one op (class_op).
  OP_CLASS = 8,
};

// A class op's kind word: OP_CLASS with its rotation count above the low byte.
__host__ __device__ inline u32 class_kind(u32 m) { return OP_CLASS | (m << 8); }
__host__ __device__ inline bool is_class(u32 kind) { return (kind & 0xffu) == OP_CLASS; }

// Rotations run by an op: 2 to 4 for a fused group's head, m for a class, else 1.
__host__ __device__ inline u32 fused_count(u32 kind) {
  if (is_class(kind)) return kind >> 8;
  return kind == OP_GATE2 ? 2u : (kind == OP_GATE3 ? 3u : (kind == OP_GATE4 ? 4u : 1u));
}

constexpr u32 GROUP_MAX = 2;    // rotations of a fused group (OP_GATE2, gate2_tiles)
constexpr u32 CLASS_MAX = 64;   // rotations of one class op (a row's class mask is one u64)
constexpr u32 CLASS_KMAX = 10;  // largest family dimension (class rotations one row anticommutes with)

struct OpDesc {
  u32 kind;
  u32 idx;  // GATE / PHASE: gate descriptor; NOISE_*: noise table index
};

template <int W>
struct GateDesc {
  GenInfo<W> g;
  double sn, cs;  // sin(angle), cos(angle) from the host libm
  u32 pivot;      // in a class: a key bit of this generator that no other
                  // generator of the class has (its family coordinate)
  u32 pad_;
};

// Device-resident state of a sweep, one per engine.
struct SweepState {
  u64 n[2];       // live rows: op k reads n[k & 1], writes n[(k + 1) & 1]
  u64 peak;       // largest live count the sweeps have seen
  u64 n_mid[2];   // live rows between the rotations of a fused op run one after the other
  u64 rec_next;   // adjoint recording: next free element of rec_idx / rec_coef
  u64 rec_key_next;  // ... next free key row of rec_keys
  u32 rec_full;   // ... the pool ran out: no op from here on is recorded
  u32 halt;       // op at which a sweep stopped for capacity, or NOT_HALTED
  u32 error;      // ERR_* bits
  u32 cur;        // row buffer holding the live rows when the sweep ended
  u32 end_op;     // first op the sweep did not run
  u32 yield_after;  // batched: 1 + the op after which the instance stops early (0 = none)
  u32 grid_stop;  // the sweep stopped at `halt` because the live count outgrew the grid (SweepArgs::grid_rows)
  u32 bar_count;  // grid barrier: groups arrived
  u32 bar_gen;    // grid barrier generation
  u64 need_rows;       // rows a class op stopped for (its output), for the host's growth
  u32 barrier_limit;   // polls a grid-barrier wait makes before it gives up (ERR_BARRIER_TIMEOUT)
  u32 lookback_limit;  // polls a tile's look-back makes before it gives up (ERR_LOOKBACK_TIMEOUT)
  static constexpr unsigned BAR_GROUPS = 16;
  struct alignas(128) Group {
    u32 count;    // blocks of this group arrived
  } bar_group[BAR_GROUPS];
};

struct SweepArgs {
  const OpDesc* ops;
  const void* gates;       // GateDesc<W>[], in op order
  u32 n_gdesc;             // gate descriptors in `gates`
  u32 pad0_;
  const double* tables;    // noise factor tables, table_len entries each
  u32 table_len;
  u32 n_units;
  u32 n_words;             // W of this propagation's keys
  u32 op_begin, op_end;    // ops [op_begin, op_end) of the sequence
  u32 cur0;                // row buffer holding the live rows at entry
  u32 epoch_base;          // tags this launch's tile statuses
  u32 max_weight;          // NO_WEIGHT_CUT if none
  u32 has_min_coeff;
  double min_coeff;
  u64 min_terms;           // TermBudget floor, 0 = none
  u64* keys[2];            // row keys, W words each, double buffered
  double* coeffs[2];
  u64* table;              // open-addressing slots: (fingerprint << 32) | row
  u64 table_mask;
  u64 table_bmask;         // ~(slots per bucket - 1): where a key's probe starts
  u64 cap;                 // rows each buffer holds
  u64 grid_rows;           // stop before an op whose live count exceeds this, 0 = never (see grid_stop)
  u64* status;             // tile look-back status words
  u32* tickets;            // per-op tile counters for many-row gates, zero at entry
  u64* hist;               // live count after each op
  u64* anti;               // anticommuting rows each gate op saw
  u64* stamps;             // %globaltimer at the end of each op
  SweepState* st;
  u32 blk_begin, blk_count;  // blocks of a batched launch that run this instance
  u32* idle_blocks;          // batched: blocks whose instance has left the launch (null: never yield)
  u32 yield_at;              // ... stop at the next op boundary once this many are idle
  // Recording for the adjoint (null: off).  Per op, from element rec_off[op]:
  // gate / phase ops store each anticommuting pre-op row's coefficient
  // (rec_coef) and the post-op row its sin branch went to, or REC_NONE
  // (rec_idx); a reclaim stores each row's new index or REC_NONE (rec_idx)
  // and its pre-op keys from row rec_key_off[op] of rec_keys.  The sweep
  // places the ops one after another from SweepState::rec_next /
  // rec_key_next, writes rec_off / rec_key_off, and stops recording (sets
  // rec_full) when the next op would not fit in rec_cap / rec_key_cap.
  u32* rec_idx;
  double* rec_coef;
  u64* rec_keys;
  u64* rec_off;
  u64* rec_key_off;
  u64 rec_cap, rec_key_cap;
  // Decisions made on the host for a launch of one op (null: the device's own
  // rules).  host_state: per input row, the emit state of its sin branch
  // (S_EMIT 0 / S_HELD 1), from a truncator plugin's keep.  host_factor: per
  // row, the noise factor (a key-reading noise model).  host_keep: per row,
  // the reclaim decision (a truncator plugin's keep_batch).
  const unsigned char* host_state;
  const double* host_factor;
  const unsigned char* host_keep;
  // Class ops (null without them): per row, the mask of class rotations it
  // anticommutes with and the slot of its family; per family owner, the rows
  // the family creates; the family table (slots (fingerprint << 32) | first
  // row, table_mask + 1 of them) and per slot (count << 32) | (~ least row).
  u64* cls_mask;
  u32* cls_slot;
  u32* cls_children;
  u64* fam_table;
  u64* fam_aux;
  // Per-op emit statistics for the verbose log (null: off), LOG_WORDS words
  // per op: branches held back by the emit check, the sum and the largest
  // |branch| of those no partner claimed (double bits), branches that went
  // out, and those that landed on an existing row.
  u64* log;
  // Failure tests (pq_engine_set_limits): block hold_block waits hold_us
  // microseconds before its first op, so that the other blocks' bounded waits
  // on it run out.  hold_us 0 = off.
  u32 hold_block, hold_us;
  // Rows per thread of a many-row gate tile (1-4; 0 = 4).
  u32 tile_items;
  u32 pad1_;
};

enum : u32 { LOG_HELD = 0, LOG_L1 = 1, LOG_MAX = 2, LOG_EMITTED = 3, LOG_HITS = 4, LOG_WORDS = 5 };

// Default wait limits (SweepState::barrier_limit / lookback_limit).
constexpr u32 DEFAULT_BARRIER_POLLS = 1u << 25;   // ~2 s with the back-off of the wait
constexpr u32 DEFAULT_LOOKBACK_POLLS = 1u << 22;  // ~0.3 s

constexpr u32 REC_NONE = 0xffffffffu;

// The reverse sweep of the adjoint over ops [op_begin, op_end) of one
// recorded segment, last op first.  lam[cur0] holds dE/dc of the rows after
// op_end - 1; each op maps it to dE/dc of its input rows in the other buffer,
// and its dE/d(angle) partial of every block goes to grad_part[op * grid + block].
struct AdjointArgs {
  const OpDesc* ops;
  const void* gates;
  const double* tables;
  u32 table_len;
  u32 n_units;
  u32 op_begin, op_end;
  u32 cur0;
  const u64* n_in;               // rows entering each op
  const u32* rec_idx;
  const double* rec_coef;
  const u64* rec_off;
  const u64* const* key_src;     // per op: keys of its input rows
  double* lam[2];
  double* grad_part;
  SweepState* st;                // barrier only
};

struct ExpectArgs {
  u64 state[64];            // basis state in key layout (Pauli: bit 2q+1; Majorana: bit 2k)
  u32 n_units;
  u32 has_min_coeff;
  double min_coeff;
  const u64* frame_images;  // readout tableau rows (2 n_units rows of W words), or null
  const int* frame_signs;   // +1 / -1 per row
  u32 frame_rows;
};

struct ExpectPartial {
  double hi, lo;    // double-double partial sum of c * trace
  double abs_sum;   // sum of |c * trace|
  u64 below;        // |c| < min_coeff
};

// Builds of the sweep kernel: for its default occupancy (MinBlocks), for six
// resident blocks per SM (1- and 2-word keys, live sets of 2^24 rows and
// more), for two (keys of at most 4 words, the one- and two-block-per-SM
// grids).  A width without the build asked for takes the default one.
enum SweepBuild : int { SWEEP_DEFAULT = 0, SWEEP_SIX = 1, SWEEP_TWO = 2 };

// Co-resident grid of the sweep kernel for this W / algebra and build: every
// SM with blocks_per_sm blocks (0 or more than fit = as many as fit).
template <int W, int ALG>
int sweep_grid(int blocks_per_sm, int build = SWEEP_DEFAULT);

template <int W, int ALG>
cudaError_t launch_sweep(const SweepArgs& a, int grid, cudaStream_t s, int build = SWEEP_DEFAULT);
// Batched sweep of instances with keys WM or WM / 2 words wide (n_words):
// args[i] describes instance i and its blk_begin / blk_count slice of the
// grid; block_inst[b] is the instance of block b.  batch_grid is its
// co-resident grid, as sweep_grid.
template <int WM, int ALG>
int batch_grid(int blocks_per_sm);
template <int WM, int ALG>
cudaError_t launch_batch_sweep(const SweepArgs* args, const u32* block_inst, int grid, cudaStream_t s);
// Cooperative launch of the reverse sweep; grid from adjoint_grid (the
// co-resident grid), grad_part holds n_ops * grid partials.
template <int W, int ALG>
int adjoint_grid();
template <int W, int ALG>
cudaError_t launch_adjoint(const AdjointArgs& a, int grid, cudaStream_t s);
// dE/dc of every row: sign * <s|frame(K)|s>, the seed of the reverse sweep.
template <int W, int ALG>
cudaError_t launch_adjoint_seed(const ExpectArgs& a, const u64* keys, u64 n, double* lam, cudaStream_t s);
// grad[g] = sum over blocks of grad_part[op * grid + b] for op = gate_ops[g]
// (NaN where gate_ops[g] < 0), in block order.
cudaError_t launch_grad_reduce(const double* grad_part, int grid, const long long* gate_ops, u64 n_gates,
                               double* grad, cudaStream_t s);
template <int W, int ALG>
cudaError_t launch_expect(const ExpectArgs& a, const u64* keys, const double* coeffs, u64 n,
                          ExpectPartial* partials, int grid, cudaStream_t s);
template <int W>
cudaError_t launch_rebuild(const u64* keys, u64 n, u64* table, u64 table_mask, u64 bucket_mask, u32* error,
                           cudaStream_t s);
template <int W>
cudaError_t launch_conjugate(const u64* keys, const double* coeffs, u64 n, const u64* frame_images,
                             const int* frame_signs, u32 frame_rows, int alg, u64* out_keys,
                             double* out_coeffs, cudaStream_t s);

}  // namespace pq
