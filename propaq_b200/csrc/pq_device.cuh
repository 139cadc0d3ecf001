// pq_device.cuh -- device-side basis algebra and key hashing of the B200
// propagation engine.
//
// Keys are W u64 words, two bits per unit, interleaved (bit 2q = x and bit
// 2q+1 = z of qubit q for Pauli; bit m = Majorana mode m).  All key logic is
// popcount / xor arithmetic on those words; no transcendental function is
// evaluated on the device (sin/cos/exp come from the host's libm, so the
// engine rounds exactly as the reference does).
#pragma once

#include <cstdint>
#include <type_traits>

namespace pq {

using u64 = unsigned long long;
using u32 = unsigned int;

constexpr u64 EVEN = 0x5555555555555555ULL;
constexpr u64 EMPTY_SLOT = ~0ULL;  // hash slot sentinel: fp 0xffffffff, row 0xffffffff
constexpr u32 NO_WEIGHT_CUT = 0xffffffffu;
constexpr u32 NOT_HALTED = 0xffffffffu;

// Error bits the kernels raise instead of hanging or faulting.
enum : u32 {
  ERR_LOOKBACK_TIMEOUT = 1u,  // a tile's predecessor never published its count
  ERR_PROBE_OVERFLOW = 2u,    // a hash probe ran past the table size
  ERR_CAPACITY = 4u,          // a write would have passed the row capacity
  ERR_BARRIER_TIMEOUT = 8u,   // a grid barrier wait expired
  ERR_CLASS_FAMILY = 16u,     // a row's family in a class op exceeded CLASS_KMAX (the host rules it out)
};

__host__ __device__ inline int mod4(int v) { return v & 3; }

__device__ __forceinline__ int popc(u64 x) { return __popcll(x); }

// splitmix64 finaliser, folded over the key's words.
__host__ __device__ __forceinline__ u64 mix64(u64 x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
template <int W>
__host__ __device__ __forceinline__ u64 key_hash(const u64* k) {
  u64 h = mix64(k[0]);
#pragma unroll
  for (int i = 1; i < W; ++i) h = mix64(h ^ k[i]);
  return h;
}

// Per-gate generator data, computed once on the host.
template <int W>
struct GenInfo {
  u64 gen[W];    // generator key (after the Clifford frame)
  u64 fold[W];   // Pauli: pair-swapped generator; Majorana: the generator
  u64 sfx[W];    // Majorana: per word, parity of generator bits strictly above each bit
  u64 carry;     // Majorana: bit w = parity of generator bits in words above w (W <= 64)
  int aux;       // Pauli: Y sites of the generator; Majorana: its length
  double sign;   // +1 / -1 carried by the generator from the frame
};

// GenInfo of generator g (W words, already conjugated through the frame) with
// frame sign `sign`; built once per rotation on the host.
template <int W>
inline GenInfo<W> make_gen_info(int alg, const u64* g, int sign) {
  auto pc = [](u64 x) { return __builtin_popcountll(x); };
  GenInfo<W> gi;
  int aux = 0;
  for (int i = 0; i < W; ++i) {
    gi.gen[i] = g[i];
    gi.fold[i] = alg == 0 ? (((g[i] & EVEN) << 1) | ((g[i] >> 1) & EVEN)) : g[i];
    aux += alg == 0 ? pc(g[i] & (g[i] >> 1) & EVEN) : pc(g[i]);
  }
  gi.aux = aux;
  gi.sign = sign < 0 ? -1.0 : 1.0;
  gi.carry = 0;
  int above = 0;
  for (int i = W - 1; i >= 0; --i) {
    u64 s = g[i] >> 1;
    for (int sh = 1; sh < 64; sh <<= 1) s ^= s >> sh;
    gi.sfx[i] = s;
    if (above) gi.carry |= 1ull << i;
    above ^= pc(g[i]) & 1;
  }
  return gi;
}

// ---------------------------------------------------------------- Pauli
// crates/pauli/src/algebra.rs:130-240
struct PauliOps {
  template <int W>
  __device__ __forceinline__ static bool anticommutes(const GenInfo<W>& g, const u64* k) {
    u64 acc = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) acc ^= k[i] & g.fold[i];
    return popc(acc) & 1;
  }
  // Phase exponent p of G*K = i^p * (G xor K) (before the generator sign).
  template <int W>
  __device__ __forceinline__ static int product_exp(const GenInfo<W>& g, const u64* k) {
    int yk = 0, yo = 0, zx = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) {
      u64 o = k[i] ^ g.gen[i];
      yk += popc(k[i] & (k[i] >> 1) & EVEN);
      yo += popc(o & (o >> 1) & EVEN);
      zx += popc((g.gen[i] >> 1) & k[i] & EVEN);
    }
    return mod4(g.aux + yk - yo + 2 * zx);
  }
  template <int W>
  __device__ __forceinline__ static u32 weight(const u64* k, u32 /*n_units*/) {
    u32 n = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) n += popc((k[i] | (k[i] >> 1)) & EVEN);
    return n;
  }
  // <s| K |s>: 0 with any x bit, else (-1)^(z bits on occupied qubits).
  // zstate has bit 2q+1 set where the state has qubit q = 1.
  template <int W>
  __device__ __forceinline__ static double trace(const u64* k, const u64* zstate, u32 /*n_units*/) {
    u64 xs = 0, par = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) {
      xs |= k[i] & EVEN;
      par ^= k[i] & zstate[i];
    }
    if (xs) return 0.0;
    return (popc(par) & 1) ? -1.0 : 1.0;
  }
};

// ------------------------------------------------------------- Majorana
// crates/majorana/src/algebra.rs:85-216, crates/majorana/src/monomial.rs:688-718
struct MajoranaOps {
  __device__ __forceinline__ static int herm(int len) { return ((len & 3) >= 2) ? 1 : 0; }
  template <int W>
  __device__ __forceinline__ static bool anticommutes(const GenInfo<W>& g, const u64* k) {
    int overlap = 0, len = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) {
      overlap += popc(k[i] & g.gen[i]);
      len += popc(k[i]);
    }
    return ((overlap + ((g.aux & 1) ? len : 0)) & 1) == 1;
  }
  // Parity of the transpositions that carry K's modes past the generator's:
  // for every mode y of K, the generator modes above y.  sfx/carry make it a
  // popcount per word.
  template <int W>
  __device__ __forceinline__ static int product_exp(const GenInfo<W>& g, const u64* k) {
    int lk = 0, lo = 0, sw = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) {
      u64 o = k[i] ^ g.gen[i];
      int pk = popc(k[i]);
      lk += pk;
      lo += popc(o);
      sw ^= (popc(k[i] & g.sfx[i]) & 1) ^ (pk & (int)((g.carry >> i) & 1ull));
    }
    return mod4(herm(g.aux) + herm(lk) - herm(lo) + 2 * (sw & 1));
  }
  // Jordan-Wigner weight: a site is non-identity if it holds exactly one
  // Majorana, or if its pair occupancy disagrees with the parity string of the
  // single Majoranas at or below it (complemented when their total is odd).
  template <int W>
  __device__ __forceinline__ static u32 weight(const u64* k, u32 n_sites) {
    int total_single = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) total_single += popc((k[i] ^ (k[i] >> 1)) & EVEN);
    const bool odd = total_single & 1;
    u32 wsum = 0;
    u64 carry = 0;  // EVEN if the singles below this word have odd parity
#pragma unroll
    for (int i = 0; i < W; ++i) {
      u64 s = (k[i] ^ (k[i] >> 1)) & EVEN;
      u64 occ = (k[i] | (k[i] >> 1)) & EVEN;
      u64 p = s;
      p ^= p << 2;
      p ^= p << 4;
      p ^= p << 8;
      p ^= p << 16;
      p ^= p << 32;
      p ^= carry;
      carry = (popc(p & (1ULL << 62)) ? EVEN : 0ULL);
      const long lo = (long)i * 32;
      const long live_sites = (long)n_sites - lo;
      u64 live = live_sites <= 0 ? 0ULL : (live_sites >= 32 ? EVEN : (EVEN & ((1ULL << (2 * live_sites)) - 1)));
      u64 str = (odd ? (p ^ EVEN) : p) & live;
      wsum += popc((s | (occ ^ str)) & live);
    }
    return wsum;
  }
  // <s| K |s> for a computational-basis determinant (algebra.rs:200-216):
  // 0 if any site holds exactly one mode, else (-1)^(pairs/2) times
  // prod (2 n_k - 1) over the paired sites.  nstate has bit 2k set where n_k = 1.
  template <int W>
  __device__ __forceinline__ static double trace(const u64* k, const u64* nstate, u32 /*n_sites*/) {
    u64 unpaired = 0;
    int paired = 0, empty_pairs = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) {
      unpaired |= (k[i] ^ (k[i] >> 1)) & EVEN;
      u64 pr = k[i] & EVEN;
      paired += popc(pr);
      empty_pairs += popc(pr & ~nstate[i]);
    }
    if (unpaired) return 0.0;
    int neg = ((paired >> 1) & 1) ^ (empty_pairs & 1);
    return neg ? -1.0 : 1.0;
  }
};

}  // namespace pq
