// pq_kernels.cuh -- kernel launch interface of the B200 propagation engine.
#pragma once

#include <cuda_runtime.h>

#include "pq_device.cuh"

namespace pq {

// Device buffers of one engine, as the kernels see them.
struct DevBufs {
  u64* keys;         // current rows, W words each (row-major)
  double* coeffs;    // current coefficients
  u64* keys_alt;     // ping-pong target of a reclaim
  double* coeffs_alt;
  u64* table;        // open-addressing slots: (fingerprint << 32) | row
  u64 table_mask;    // slots - 1
  u64 cap;           // rows each buffer holds
  u64* status;       // tile look-back status words
  Ctl* ctl;
  u64* hist;         // live count after each op
  u64* anti;         // anticommuting rows seen by each gate op
};

// Per-gate arguments.
template <int W>
struct GateArgs {
  GenInfo<W> g;
  double sn, cs;        // sin(angle), cos(angle) from the host libm
  u32 max_weight;       // NO_WEIGHT_CUT if none
  u32 has_min_coeff;
  double min_coeff;
  u64 min_terms;        // TermBudget floor, 0 = none
  u32 n_units;
  u32 op;               // op index (capacity halts and the per-op history)
};

struct NoiseArgs {
  const double* factors;  // factor by weight (device)
  u32 table_len;
  u32 n_units;
  u32 max_weight;         // reclaim predicate; NO_WEIGHT_CUT if none
  u32 has_min_coeff;
  double min_coeff;
  u32 compact;            // 0: scale only (no truncation configured)
  u32 op;
};

struct ExpectArgs {
  u64 state[64];          // basis state in key layout (Pauli: bit 2q+1; Majorana: bit 2k)
  u32 n_units;
  u32 has_min_coeff;
  double min_coeff;
  const u64* frame_images;  // readout tableau rows (2 n_units rows of W words), or null
  const int* frame_signs;   // +1 / -1 per row
  u32 frame_rows;
};

struct ExpectPartial {
  double hi, lo;      // double-double partial sum of c * trace
  double abs_sum;     // sum of |c * trace|
  u64 below;          // |c| < min_coeff
};

int launch_blocks();  // persistent grid size for the current device

template <int W, int ALG>
cudaError_t launch_gate(const GateArgs<W>& a, const DevBufs& b, int grid, cudaStream_t s);
template <int W, int ALG>
cudaError_t launch_phase_only(const GateArgs<W>& a, const DevBufs& b, int grid, cudaStream_t s);
template <int W, int ALG>
cudaError_t launch_noise(const NoiseArgs& a, const DevBufs& b, int grid, cudaStream_t s);
template <int W, int ALG>
cudaError_t launch_expect(const ExpectArgs& a, const DevBufs& b, ExpectPartial* partials, int grid,
                          cudaStream_t s);
template <int W>
cudaError_t launch_rebuild(const DevBufs& b, int grid, cudaStream_t s);
template <int W>
cudaError_t launch_conjugate(const DevBufs& b, const u64* frame_images, const int* frame_signs,
                             u32 frame_rows, int alg, u64* out_keys, double* out_coeffs, u64 n,
                             cudaStream_t s);

}  // namespace pq
