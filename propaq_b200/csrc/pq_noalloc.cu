// pq_noalloc.cu -- pq_expectation_noalloc: the expectation reduction of
// expect_kernel for callers that may not allocate device memory.
//
// Some programs that embed this library own every byte of device memory
// themselves: frameworks that reserve (almost) the whole GPU up front for
// their own caching allocators (a JAX process with memory preallocation, a
// serving engine that sizes its KV cache to the remaining memory), or
// applications with a fixed device-memory budget set at start-up.  A
// cudaMalloc issued from inside such a program fails or breaks the owner's
// accounting.  This entry point therefore allocates nothing: it stages the
// caller's terms into a file-scope static __device__ array, reduces them there
// and copies the scalar back.  The array (PQ_NOALLOC_SCRATCH_BYTES, 16 MiB)
// is created when this module is first loaded on a device and is held by that
// device until the process exits.
//
// Set-up: every call resolves the array's device address with
// cudaGetSymbolAddress while the caller's device is current, so the address
// is right for whatever context is current -- after a cudaDeviceReset (which
// reloads the module, possibly elsewhere) as well as in a context the caller
// created itself.  The lookup allocates nothing.  The module (and with it the
// 16 MiB array) is loaded on a device at the first call there (or when the
// library is loaded, with CUDA_MODULE_LOADING=EAGER): make that first call
// before the program reserves its device memory, and before any stream
// capture begins.
//
// Sharing: every call on a device uses the same array, which keeps the last
// call's contents.  Calls issued concurrently on one device (e.g. from two host
// threads) overlap on the GPU and race on the array; serialise them.  Nothing
// in the array needs to start at zero: each call writes every slot it later
// reads (its staged terms, one partial per block, the result slot).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/propaq_cuda.h"
#include "pq_device.cuh"

namespace {

using pq::u32;
using pq::u64;

constexpr int NA_BLOCK = 256;
constexpr int NA_MAX_BLOCKS = 512;
constexpr size_t NA_PARTIALS_BYTES = NA_MAX_BLOCKS * 16;  // (hi, lo) per block
constexpr size_t NA_RESULT_BYTES = 256;
constexpr size_t NA_TERMS_OFFSET = NA_PARTIALS_BYTES + NA_RESULT_BYTES;
static __device__ __align__(256) unsigned char pq_noalloc_scratch[PQ_NOALLOC_SCRATCH_BYTES];

thread_local std::string g_error;

__device__ __forceinline__ void na_two_sum(double a, double b, double& s, double& e) {
  s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}
__device__ __forceinline__ void na_dd_add(double& hi, double& lo, double v) {
  double s, e;
  na_two_sum(hi, v, s, e);
  e = __dadd_rn(e, lo);
  na_two_sum(s, e, hi, lo);
}

struct NaState {
  u64 words[64];  // basis state in key layout (Pauli: bit 2q+1; Majorana: bit 2k)
};

// Per-block double-double partial sums of c * <s|K|s>.
template <int W, int ALG>
__global__ void __launch_bounds__(NA_BLOCK) na_expect_kernel(const NaState s, u32 n_units, const u64* keys,
                                                             const double* coeffs, u64 n, double* partials) {
  double hi = 0, lo = 0;
  for (u64 r = (u64)blockIdx.x * NA_BLOCK + threadIdx.x; r < n; r += (u64)gridDim.x * NA_BLOCK) {
    u64 key[W];
#pragma unroll
    for (int i = 0; i < W; ++i) key[i] = keys[r * W + i];
    double tr;
    if constexpr (ALG == 0)
      tr = pq::PauliOps::trace<W>(key, s.words, n_units);
    else
      tr = pq::MajoranaOps::trace<W>(key, s.words, n_units);
    const double v = __dmul_rn(coeffs[r], tr);
    if (v != 0.0) na_dd_add(hi, lo, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ohi = __shfl_xor_sync(0xffffffffu, hi, o), olo = __shfl_xor_sync(0xffffffffu, lo, o);
    na_dd_add(hi, lo, ohi);
    na_dd_add(hi, lo, olo);
  }
  __shared__ double shi[NA_BLOCK / 32], slo[NA_BLOCK / 32];
  if ((threadIdx.x & 31) == 0) {
    shi[threadIdx.x >> 5] = hi;
    slo[threadIdx.x >> 5] = lo;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double h = 0, l = 0;
    for (int w = 0; w < NA_BLOCK / 32; ++w) {
      na_dd_add(h, l, shi[w]);
      na_dd_add(h, l, slo[w]);
    }
    partials[2 * blockIdx.x] = h;
    partials[2 * blockIdx.x + 1] = l;
  }
}

// Folds the block partials (one thread, in block order) into result[0].
__global__ void na_finalize_kernel(const double* partials, int n_blocks, double* result) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double h = 0, l = 0;
  for (int b = 0; b < n_blocks; ++b) {
    na_dd_add(h, l, partials[2 * b]);
    na_dd_add(h, l, partials[2 * b + 1]);
  }
  result[0] = __dadd_rn(h, l);
}

template <int W, int ALG>
cudaError_t na_launch(const NaState& s, u32 n_units, const u64* keys, const double* coeffs, u64 n, double* partials,
                      int blocks) {
  na_expect_kernel<W, ALG><<<blocks, NA_BLOCK>>>(s, n_units, keys, coeffs, n, partials);
  return cudaGetLastError();
}

int na_fail(int code, const std::string& m) {
  g_error = m;
  return code;
}

int pq_expectation_noalloc_impl(uint32_t basis_kind, uint32_t n_units, const uint64_t* keys, const double* coeffs,
                                size_t n_terms, const uint64_t* diag_state, size_t diag_words, double* out_value);

}  // namespace

extern "C" {

int pq_expectation_noalloc(uint32_t basis_kind, uint32_t n_units, const uint64_t* keys, const double* coeffs,
                           size_t n_terms, const uint64_t* diag_state, size_t diag_words, double* out_value,
                           char* err, size_t err_len) {
  int rc = pq_expectation_noalloc_impl(basis_kind, n_units, keys, coeffs, n_terms, diag_state, diag_words, out_value);
  if (rc != PQ_OK && err && err_len) snprintf(err, err_len, "%s", g_error.c_str());
  return rc;
}

}  // extern "C"

namespace {

int pq_expectation_noalloc_impl(uint32_t basis_kind, uint32_t n_units, const uint64_t* keys, const double* coeffs,
                                size_t n_terms, const uint64_t* diag_state, size_t diag_words, double* out_value) {
  g_error.clear();
  if (!out_value || (n_terms && (!keys || !coeffs)))
    return na_fail(PQ_ERR_INVALID, "pq_expectation_noalloc: null argument");
  if (basis_kind > 1) return na_fail(PQ_ERR_INVALID, "basis_kind must be 0 (Pauli) or 1 (Majorana)");
  const uint32_t W = pq_words_for_units(n_units);
  if (W == 0 || W > 8)
    return na_fail(PQ_ERR_INVALID, "pq_expectation_noalloc: " + std::to_string(n_units) +
                                       " units is beyond the 256-unit limit of this entry point");
  const size_t need = NA_TERMS_OFFSET + n_terms * (8 * (size_t)W + 8);
  if (need > PQ_NOALLOC_SCRATCH_BYTES)
    return na_fail(PQ_ERR_INVALID, "pq_expectation_noalloc: " + std::to_string(n_terms) + " terms of " +
                                       std::to_string(W) + " words need " + std::to_string(need) +
                                       " bytes of device scratch; the static scratch holds " +
                                       std::to_string((size_t)PQ_NOALLOC_SCRATCH_BYTES) + " bytes");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return na_fail(PQ_ERR_CUDA, "pq_expectation_noalloc: no current CUDA device");
  }
  // The array's address in the current context, looked up on every call (see
  // the set-up note above); a host-side name of the array is not an address
  // the device can use.
  void* base = nullptr;
  e = cudaGetSymbolAddress(&base, pq_noalloc_scratch);
  if (e != cudaSuccess || !base) {
    cudaGetLastError();
    return na_fail(PQ_ERR_CUDA, std::string("pq_expectation_noalloc: cudaGetSymbolAddress failed: ") +
                                    cudaGetErrorString(e));
  }
  unsigned char* b = static_cast<unsigned char*>(base);
  double* partials = reinterpret_cast<double*>(b);
  double* result = reinterpret_cast<double*>(b + NA_PARTIALS_BYTES);
  u64* d_keys = reinterpret_cast<u64*>(b + NA_TERMS_OFFSET);
  double* d_coeffs = reinterpret_cast<double*>(b + NA_TERMS_OFFSET + n_terms * 8 * (size_t)W);

  NaState s;
  std::memset(&s, 0, sizeof s);
  for (u32 u = 0; diag_state && u < n_units; ++u) {
    const u64 bit = (u / 64 < diag_words) ? (diag_state[u / 64] >> (u % 64)) & 1 : 0;
    if (!bit) continue;
    const u32 pos = basis_kind == 0 ? 2 * u + 1 : 2 * u;
    s.words[pos / 64] |= 1ULL << (pos % 64);
  }
  if (n_terms) {
    if ((e = cudaMemcpy(d_keys, keys, n_terms * 8 * (size_t)W, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(d_coeffs, coeffs, n_terms * 8, cudaMemcpyHostToDevice)) != cudaSuccess)
      return na_fail(PQ_ERR_CUDA, std::string("pq_expectation_noalloc: staging copy failed: ") + cudaGetErrorString(e));
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int blocks = (int)((n_terms + NA_BLOCK - 1) / NA_BLOCK);
  if (blocks > 2 * sms) blocks = 2 * sms;
  if (blocks > NA_MAX_BLOCKS) blocks = NA_MAX_BLOCKS;
  if (blocks < 1) blocks = 1;
  const u32 alg = basis_kind;
  switch (W * 2 + alg) {
    case 2: e = na_launch<1, 0>(s, n_units, d_keys, d_coeffs, n_terms, partials, blocks); break;
    case 3: e = na_launch<1, 1>(s, n_units, d_keys, d_coeffs, n_terms, partials, blocks); break;
    case 4: e = na_launch<2, 0>(s, n_units, d_keys, d_coeffs, n_terms, partials, blocks); break;
    case 5: e = na_launch<2, 1>(s, n_units, d_keys, d_coeffs, n_terms, partials, blocks); break;
    case 8: e = na_launch<4, 0>(s, n_units, d_keys, d_coeffs, n_terms, partials, blocks); break;
    case 9: e = na_launch<4, 1>(s, n_units, d_keys, d_coeffs, n_terms, partials, blocks); break;
    case 16: e = na_launch<8, 0>(s, n_units, d_keys, d_coeffs, n_terms, partials, blocks); break;
    case 17: e = na_launch<8, 1>(s, n_units, d_keys, d_coeffs, n_terms, partials, blocks); break;
    default: return na_fail(PQ_ERR_INVALID, "pq_expectation_noalloc: no kernel for " + std::to_string(W) + " key words");
  }
  if (e != cudaSuccess)
    return na_fail(PQ_ERR_CUDA, std::string("pq_expectation_noalloc: launch failed: ") + cudaGetErrorString(e));
  na_finalize_kernel<<<1, 32>>>(partials, blocks, result);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return na_fail(PQ_ERR_CUDA, std::string("pq_expectation_noalloc: launch failed: ") + cudaGetErrorString(e));
  if ((e = cudaMemcpy(out_value, result, sizeof(double), cudaMemcpyDeviceToHost)) != cudaSuccess)
    return na_fail(PQ_ERR_CUDA, std::string("pq_expectation_noalloc: result copy failed: ") + cudaGetErrorString(e));
  return PQ_OK;
}

}  // namespace
