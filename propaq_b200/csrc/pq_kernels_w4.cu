// The engine's kernels for 4-word keys (65-128 units), compiled in a
// translation unit of their own so that the key widths build in parallel.
#define PQ_ONLY_WIDTH 4
#include "pq_kernels.cu"
