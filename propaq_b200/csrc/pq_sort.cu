// pq_sort.cu -- LSD radix sort of term rows by key, and the segmented sum
// that folds duplicate keys.
//
// Rows are W 64-bit key words with an f64 coefficient; the order is the key's
// value as a 64W-bit integer (word W-1 most significant).  Each pass sorts by
// one 8-bit digit, stably, so after the passes from the least to the most
// significant digit the rows are in key order and rows with equal keys keep
// their input order.  A pass whose digit is the same in every row changes
// nothing and is skipped: a counting kernel per key word first tallies its
// eight digit positions, and the host reads that tally back.
//
// A pass is three kernels:
//   digit_count    per block, the rows of its tile holding each digit value;
//   count_scan     one block: the exclusive scan of those counts taken digit
//                  major (every block's count of digit 0, then of digit 1 ...),
//                  which is where each (digit, block) run starts in the output;
//   digit_scatter  per block, its tile again, 256 rows at a time: a row's place
//                  is its run's start plus the rows of equal digit before it
//                  (earlier 256-row chunks, earlier warps, earlier lanes:
//                  __match_any_sync finds the lanes of equal digit).
//
// fold_sorted sums runs of equal keys of a sorted array, each run from its
// first row to its last one after the other, so the sums round as a
// left-to-right loop over the input order does.
#include <cuda_runtime.h>

#include <vector>

#include "pq_sort.cuh"

namespace pq {

namespace {

constexpr int SORT_BLOCK = 256;
constexpr int SORT_CHUNKS = 8;                       // 256-row chunks per tile
constexpr int SORT_TILE = SORT_BLOCK * SORT_CHUNKS;  // rows per block per pass
constexpr int SORT_WARPS = SORT_BLOCK / 32;
constexpr unsigned FULL_MASK = 0xffffffffu;

template <int W>
__device__ __forceinline__ u32 digit_of(const u64* keys, u64 row, int pass) {
  return (u32)((keys[row * W + (pass >> 3)] >> (8 * (pass & 7))) & 0xffu);
}

// The 8 digit positions of key word w of every row at once:
// tally[(8 w + byte) * 256 + digit].
template <int W>
__global__ void __launch_bounds__(SORT_BLOCK) digit_tally_kernel(const u64* keys, u64 n, int w, u32* tally) {
  __shared__ u32 t[8 * 256];
  for (int i = threadIdx.x; i < 8 * 256; i += SORT_BLOCK) t[i] = 0;
  __syncthreads();
  for (u64 r = (u64)blockIdx.x * SORT_BLOCK + threadIdx.x; r < n; r += (u64)gridDim.x * SORT_BLOCK) {
    const u64 k = keys[r * W + w];
#pragma unroll
    for (int b = 0; b < 8; ++b) atomicAdd(&t[b * 256 + ((k >> (8 * b)) & 0xffu)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 8 * 256; i += SORT_BLOCK)
    if (t[i]) atomicAdd(&tally[w * 8 * 256 + i], t[i]);
}

template <int W>
__global__ void __launch_bounds__(SORT_BLOCK) digit_count_kernel(const u64* keys, u64 n, int pass, u32* counts,
                                                                 u32 nblk) {
  __shared__ u32 c[256];
  c[threadIdx.x] = 0;
  __syncthreads();
  const u64 base = (u64)blockIdx.x * SORT_TILE;
  for (int i = 0; i < SORT_CHUNKS; ++i) {
    const u64 r = base + (u64)i * SORT_BLOCK + threadIdx.x;
    if (r < n) atomicAdd(&c[digit_of<W>(keys, r, pass)], 1u);
  }
  __syncthreads();
  counts[(u64)threadIdx.x * nblk + blockIdx.x] = c[threadIdx.x];
}

// Exclusive scan of m counts in place, one block of 1024 threads: each thread
// sums a contiguous stretch, the block scans the stretch sums, each thread
// rewrites its stretch.
__global__ void __launch_bounds__(1024) count_scan_kernel(u32* counts, u64 m) {
  __shared__ u32 part[1024];
  const u64 per = (m + 1023) / 1024;
  const u64 lo = (u64)threadIdx.x * per, hi = lo + per < m ? lo + per : m;
  u32 s = 0;
  for (u64 i = lo; i < hi; ++i) s += counts[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const u32 v = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0u;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  u32 run = part[threadIdx.x] - s;
  for (u64 i = lo; i < hi; ++i) {
    const u32 v = counts[i];
    counts[i] = run;
    run += v;
  }
}

template <int W>
__global__ void __launch_bounds__(SORT_BLOCK) digit_scatter_kernel(const u64* keys, const double* coeffs, u64 n,
                                                                   int pass, const u32* offsets, u32 nblk,
                                                                   u64* keys_out, double* coeffs_out) {
  __shared__ u32 run[256];                // next output place of each digit for this block
  __shared__ u32 wcnt[SORT_WARPS][256];   // rows of each digit in each warp of the chunk
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  run[threadIdx.x] = offsets[(u64)threadIdx.x * nblk + blockIdx.x];
  for (int w = 0; w < SORT_WARPS; ++w) wcnt[w][threadIdx.x] = 0;
  __syncthreads();
  const u64 base = (u64)blockIdx.x * SORT_TILE;
  for (int i = 0; i < SORT_CHUNKS; ++i) {
    const u64 r = base + (u64)i * SORT_BLOCK + threadIdx.x;
    const bool live = r < n;
    const u32 d = live ? digit_of<W>(keys, r, pass) : 256u + (u32)lane;  // dead lanes match nobody
    const unsigned peers = __match_any_sync(FULL_MASK, d);
    const u32 rank = __popc(peers & ((1u << lane) - 1u));
    if (live && rank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    if (live) {
      u32 pos = run[d] + rank;
      for (int w = 0; w < warp; ++w) pos += wcnt[w][d];
#pragma unroll
      for (int k = 0; k < W; ++k) keys_out[(u64)pos * W + k] = keys[r * W + k];
      coeffs_out[pos] = coeffs[r];
    }
    __syncthreads();
    u32 add = 0;
    for (int w = 0; w < SORT_WARPS; ++w) {
      add += wcnt[w][threadIdx.x];
      wcnt[w][threadIdx.x] = 0;
    }
    run[threadIdx.x] += add;
    __syncthreads();
  }
}

// 1 where a sorted row starts a run of equal keys.
template <int W>
__global__ void run_heads_kernel(const u64* keys, u64 n, u32* head) {
  for (u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (u64)gridDim.x * blockDim.x) {
    bool h = r == 0;
    if (!h)
#pragma unroll
      for (int k = 0; k < W; ++k) h |= keys[r * W + k] != keys[(r - 1) * W + k];
    head[r] = h ? 1u : 0u;
  }
}

// Each run's first row writes the run's key and its coefficients' sum, in
// input order, at the run's index (the exclusive scan of the heads).
template <int W>
__global__ void fold_runs_kernel(const u64* keys, const double* coeffs, u64 n, const u32* head,
                                 const u32* run_index, u64* keys_out, double* coeffs_out) {
  for (u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (u64)gridDim.x * blockDim.x) {
    if (!head[r]) continue;
    double s = coeffs[r];
    for (u64 j = r + 1; j < n && !head[j]; ++j) s = __dadd_rn(s, coeffs[j]);
    const u64 o = run_index[r];
#pragma unroll
    for (int k = 0; k < W; ++k) keys_out[o * W + k] = keys[r * W + k];
    coeffs_out[o] = s;
  }
}

inline int grid_for(u64 n, int block) {
  const u64 b = (n + block - 1) / block;
  return (int)(b < 4096 ? (b ? b : 1) : 4096);
}

}  // namespace

u64 sort_scratch_words(u64 n, int W) {
  const u64 nblk = (n + SORT_TILE - 1) / SORT_TILE;
  return 256 * (nblk ? nblk : 1) / 2 + 1 + (u64)8 * W * 256 / 2 + n * (u64)W + n;
}

template <int W>
cudaError_t sort_rows(const u64* keys, const double* coeffs, u64 n, u64* keys_out, double* coeffs_out,
                      u64* scratch, cudaStream_t s, u64* launches) {
  if (n == 0) return cudaSuccess;
  const u32 nblk = (u32)((n + SORT_TILE - 1) / SORT_TILE);
  const u64 m = 256ull * nblk;
  // scratch: counts (m u32), tally (8W x 256 u32), then a second key / coefficient buffer
  u32* counts = reinterpret_cast<u32*>(scratch);
  u32* tally = counts + ((m + 1) & ~1ull);
  u64* tk = scratch + ((m + 1) & ~1ull) / 2 + (u64)8 * W * 256 / 2;
  double* tc = reinterpret_cast<double*>(tk + n * W);
  cudaError_t e;
  if ((e = cudaMemsetAsync(tally, 0, sizeof(u32) * 8 * W * 256, s)) != cudaSuccess) return e;
  for (int w = 0; w < W; ++w) {
    digit_tally_kernel<W><<<grid_for(n, SORT_BLOCK), SORT_BLOCK, 0, s>>>(keys, n, w, tally);
    ++*launches;
  }
  std::vector<u32> h_tally(8 * W * 256);
  if ((e = cudaMemcpyAsync(h_tally.data(), tally, h_tally.size() * 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return e;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  // the passes that move rows: a digit position where the rows differ
  int passes[8 * W];
  int np = 0;
  for (int p = 0; p < 8 * W; ++p) {
    bool constant = false;
    for (int d = 0; d < 256; ++d) constant |= h_tally[p * 256 + d] == n;
    if (!constant) passes[np++] = p;
  }
  // ping-pong so that the last pass lands in keys_out / coeffs_out
  const u64* src_k = keys;
  const double* src_c = coeffs;
  for (int i = 0; i < np; ++i) {
    const bool to_out = ((np - 1 - i) & 1) == 0;
    u64* dk = to_out ? keys_out : tk;
    double* dc = to_out ? coeffs_out : tc;
    digit_count_kernel<W><<<nblk, SORT_BLOCK, 0, s>>>(src_k, n, passes[i], counts, nblk);
    count_scan_kernel<<<1, 1024, 0, s>>>(counts, m);
    digit_scatter_kernel<W><<<nblk, SORT_BLOCK, 0, s>>>(src_k, src_c, n, passes[i], counts, nblk, dk, dc);
    *launches += 3;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    src_k = dk;
    src_c = dc;
  }
  if (np == 0) {  // already in order (one key, or all keys equal)
    if ((e = cudaMemcpyAsync(keys_out, keys, n * W * 8, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(coeffs_out, coeffs, n * 8, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

template <int W>
cudaError_t fold_sorted(const u64* keys, const double* coeffs, u64 n, u64* keys_out, double* coeffs_out,
                        u32* head, u64* n_out, u64* scratch, cudaStream_t s, u64* launches) {
  if (n == 0) {
    *n_out = 0;
    return cudaSuccess;
  }
  cudaError_t e;
  run_heads_kernel<W><<<grid_for(n, 256), 256, 0, s>>>(keys, n, head);
  // run index of each row: the exclusive scan of the heads (one block)
  u32* idx = reinterpret_cast<u32*>(scratch);
  if ((e = cudaMemcpyAsync(idx, head, n * 4, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
  count_scan_kernel<<<1, 1024, 0, s>>>(idx, n);
  fold_runs_kernel<W><<<grid_for(n, 256), 256, 0, s>>>(keys, coeffs, n, head, idx, keys_out, coeffs_out);
  *launches += 3;
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  u32 last_idx = 0, last_head = 0;
  if ((e = cudaMemcpyAsync(&last_idx, idx + n - 1, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(&last_head, head + n - 1, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
  *n_out = (u64)last_idx + last_head;
  return cudaGetLastError();
}

#define PQ_SORT_INSTANTIATE(Wv)                                                                                  \
  template cudaError_t sort_rows<Wv>(const u64*, const double*, u64, u64*, double*, u64*, cudaStream_t, u64*); \
  template cudaError_t fold_sorted<Wv>(const u64*, const double*, u64, u64*, double*, u32*, u64*, u64*,         \
                                       cudaStream_t, u64*);
PQ_SORT_INSTANTIATE(1)
PQ_SORT_INSTANTIATE(2)
PQ_SORT_INSTANTIATE(4)
PQ_SORT_INSTANTIATE(8)
PQ_SORT_INSTANTIATE(16)
PQ_SORT_INSTANTIATE(32)
PQ_SORT_INSTANTIATE(64)

}  // namespace pq
