// pq_sort.cuh -- radix sort of term rows by key and the folding of equal keys
// (pq_sort.cu).
#pragma once

#include <cuda_runtime.h>

#include "pq_device.cuh"

namespace pq {

// u64 words of scratch sort_rows / fold_sorted need for n rows of W words.
u64 sort_scratch_words(u64 n, int W);

// Stable sort of n rows (keys, coeffs) by key value into keys_out /
// coeffs_out (distinct from the inputs; the inputs are left as they were).
// Synchronises the stream once (to skip the digit positions where all keys
// agree).  launches counts the kernels it ran.
template <int W>
cudaError_t sort_rows(const u64* keys, const double* coeffs, u64 n, u64* keys_out, double* coeffs_out,
                      u64* scratch, cudaStream_t s, u64* launches);

// Rows sorted by key: each run of equal keys becomes one row, its
// coefficients summed from the first to the last (input order, as stable
// sorting keeps it).  head holds n u32; *n_out receives the row count
// (synchronises the stream).
template <int W>
cudaError_t fold_sorted(const u64* keys, const double* coeffs, u64 n, u64* keys_out, double* coeffs_out,
                        u32* head, u64* n_out, u64* scratch, cudaStream_t s, u64* launches);

}  // namespace pq
