// The engine's kernels for 16-word keys (257-512 units), compiled in a
// translation unit of their own so that the key widths build in parallel.
#define PQ_ONLY_WIDTH 16
#include "pq_kernels.cu"
