// The engine's Majorana kernels for 32-word keys (513-1024 units), compiled in
// a translation unit of their own so that the key widths and algebras build
// in parallel.
#define PQ_ONLY_WIDTH 32
#define PQ_ONLY_ALG 1
#include "pq_kernels.cu"
