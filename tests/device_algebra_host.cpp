// The engine's device algebra (propaq_b200/csrc/pq_device.cuh: PauliOps,
// MajoranaOps, make_gen_info) compiled for the host with g++, so that CPU
// tests can hold the very formulas the kernels run against the reference's
// known answers and against the oracle.  Built into a shared library by
// test_algebra_known_answers.py; every entry point takes keys of n_words
// (1, 2, 4 or 8) 64-bit words in the interleaved layout.
#define __host__
#define __device__
#define __forceinline__ inline
static inline int __popcll(unsigned long long x) { return __builtin_popcountll(x); }

#include "../propaq_b200/csrc/pq_device.cuh"

using pq::u32;
using pq::u64;

namespace {

template <class F>
auto by_width(u32 W, F&& f) {
  switch (W) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 4: return f(std::integral_constant<int, 4>{});
    default: return f(std::integral_constant<int, 8>{});
  }
}

}  // namespace

extern "C" {

// 1 if key anticommutes with generator gen.
int da_anticommutes(u32 alg, u32 n_words, const u64* gen, const u64* key) {
  return by_width(n_words, [&](auto w) {
    constexpr int W = decltype(w)::value;
    const pq::GenInfo<W> g = pq::make_gen_info<W>((int)alg, gen, 1);
    return alg == 0 ? (int)pq::PauliOps::anticommutes<W>(g, key) : (int)pq::MajoranaOps::anticommutes<W>(g, key);
  });
}

// Phase exponent p of gen * key = i^p (gen xor key), written to *child.
int da_product(u32 alg, u32 n_words, const u64* gen, const u64* key, u64* child) {
  for (u32 i = 0; i < n_words; ++i) child[i] = gen[i] ^ key[i];
  return by_width(n_words, [&](auto w) {
    constexpr int W = decltype(w)::value;
    const pq::GenInfo<W> g = pq::make_gen_info<W>((int)alg, gen, 1);
    return alg == 0 ? pq::PauliOps::product_exp<W>(g, key) : pq::MajoranaOps::product_exp<W>(g, key);
  });
}

u32 da_weight(u32 alg, u32 n_units, u32 n_words, const u64* key) {
  return by_width(n_words, [&](auto w) {
    constexpr int W = decltype(w)::value;
    return alg == 0 ? pq::PauliOps::weight<W>(key, n_units) : pq::MajoranaOps::weight<W>(key, n_units);
  });
}

// <s|key|s> for the basis state given as one bit per unit (diag_words words).
double da_trace(u32 alg, u32 n_units, u32 n_words, const u64* key, const u64* diag, u32 diag_words) {
  u64 s[64] = {0};
  for (u32 u = 0; u < n_units; ++u) {
    const u64 bit = (u / 64 < diag_words) ? (diag[u / 64] >> (u % 64)) & 1 : 0;
    if (!bit) continue;
    const u32 pos = alg == 0 ? 2 * u + 1 : 2 * u;
    s[pos / 64] |= 1ULL << (pos % 64);
  }
  return by_width(n_words, [&](auto w) {
    constexpr int W = decltype(w)::value;
    return alg == 0 ? pq::PauliOps::trace<W>(key, s, n_units) : pq::MajoranaOps::trace<W>(key, s, n_units);
  });
}

}  // extern "C"
