// The engine's kernels for 8-word keys (129-256 units), compiled in a
// translation unit of their own so that the key widths build in parallel.
#define PQ_ONLY_WIDTH 8
#include "pq_kernels.cu"
