// The engine's Majorana kernels for 64-word keys (1025-2048 units), compiled in
// a translation unit of their own so that the key widths and algebras build
// in parallel.
#define PQ_ONLY_WIDTH 64
#define PQ_ONLY_ALG 1
#include "pq_kernels.cu"
