// The engine's kernels for 32-word keys (513-1024 units), compiled in a
// translation unit of their own so that the key widths build in parallel.
#define PQ_ONLY_WIDTH 32
#include "pq_kernels.cu"
