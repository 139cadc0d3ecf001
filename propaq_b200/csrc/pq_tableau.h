// pq_tableau.h -- host-side key algebra and the deferred Clifford frame.
//
// Host-only C++ (no CUDA): the engine includes it, and a CPU test compiles it
// with g++ to check the frame's rotation update against the full tableau
// composition.  Keys are interleaved: unit q occupies bits 2q (X, or the
// first Majorana mode of site q) and 2q+1 (Z, or the second mode), W 64-bit
// words per key.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace pqh {

using u64 = unsigned long long;  // the engine's key word type
using u32 = unsigned int;

inline int hpopc(u64 x) { return __builtin_popcountll(x); }
constexpr u64 EVEN = 0x5555555555555555ULL;
constexpr int MAX_WORDS = 64;

// ------------------------------------------------------------ host algebra
// Phase exponent p of G*K = i^p (G xor K); the same formulas as the device
// (crates/pauli/src/algebra.rs:206-213, crates/majorana/src/algebra.rs:180-193).
inline int host_product_exp(int alg, int W, const u64* g, const u64* k) {
  if (alg == 0) {
    int yg = 0, yk = 0, yo = 0, zx = 0;
    for (int i = 0; i < W; ++i) {
      u64 o = k[i] ^ g[i];
      yg += hpopc(g[i] & (g[i] >> 1) & EVEN);
      yk += hpopc(k[i] & (k[i] >> 1) & EVEN);
      yo += hpopc(o & (o >> 1) & EVEN);
      zx += hpopc((g[i] >> 1) & k[i] & EVEN);
    }
    return (yg + yk - yo + 2 * zx) & 3;
  }
  int lg = 0, lk = 0, lo = 0, sw = 0;
  int above = 0;
  for (int i = W - 1; i >= 0; --i) {
    u64 o = k[i] ^ g[i];
    int pg = hpopc(g[i]), pk = hpopc(k[i]);
    lg += pg;
    lk += pk;
    lo += hpopc(o);
    u64 s = g[i] >> 1;
    for (int sh = 1; sh < 64; sh <<= 1) s ^= s >> sh;
    sw ^= (hpopc(k[i] & s) & 1) ^ (pk & above);
    above ^= pg & 1;
  }
  auto herm = [](int l) { return ((l & 3) >= 2) ? 1 : 0; };
  return (herm(lg) + herm(lk) - herm(lo) + 2 * (sw & 1)) & 3;
}
inline bool host_anticommutes(int alg, int W, const u64* g, const u64* k) {
  if (alg == 0) {
    u64 acc = 0;
    for (int i = 0; i < W; ++i) acc ^= k[i] & (((g[i] & EVEN) << 1) | ((g[i] >> 1) & EVEN));
    return hpopc(acc) & 1;
  }
  int ov = 0, lg = 0, lk = 0;
  for (int i = 0; i < W; ++i) {
    ov += hpopc(k[i] & g[i]);
    lg += hpopc(g[i]);
    lk += hpopc(k[i]);
  }
  return ((ov + ((lg & 1) ? lk : 0)) & 1) == 1;
}
inline int host_support(int W, const u64* k) {
  int n = 0;
  for (int i = 0; i < W; ++i) n += hpopc((k[i] | (k[i] >> 1)) & EVEN);
  return n;
}
inline u32 host_weight(int alg, int W, const u64* k, u32 n_units) {
  if (alg == 0) return (u32)host_support(W, k);
  int total = 0;
  for (int i = 0; i < W; ++i) total += hpopc((k[i] ^ (k[i] >> 1)) & EVEN);
  bool odd = total & 1;
  u32 w = 0;
  u64 carry = 0;
  for (int i = 0; i < W; ++i) {
    u64 s = (k[i] ^ (k[i] >> 1)) & EVEN, occ = (k[i] | (k[i] >> 1)) & EVEN, p = s;
    for (int sh = 2; sh < 64; sh <<= 1) p ^= p << sh;
    p ^= carry;
    carry = (p >> 62) & 1 ? EVEN : 0;
    long live_sites = (long)n_units - (long)i * 32;
    u64 live = live_sites <= 0 ? 0 : (live_sites >= 32 ? EVEN : (EVEN & ((1ULL << (2 * live_sites)) - 1)));
    u64 str = (odd ? (p ^ EVEN) : p) & live;
    w += hpopc((s | (occ ^ str)) & live);
  }
  return w;
}

// Sign of the image of an anticommuting key K under a Clifford rotation of
// generator G with sin(angle) = sn: G K = i^p (G xor K) with p odd, and the
// rotated key is sn * (-Im i^p) (G xor K) (tableau.rs:180-209 for unit keys;
// the same conjugation formula holds for every key).
inline int rotated_sign(double sn, int p) {
  const double nim = p == 1 ? -1.0 : (p == 3 ? 1.0 : 0.0);
  return sn * nim < 0 ? -1 : 1;
}

// Calls f(p) for every unit bit p < lim that can anticommute with gen: for a
// Pauli generator only the X and Z bits of the qubits it acts on (a unit on
// any other qubit commutes with it), for a Majorana generator every bit.
template <class F>
inline void for_candidate_units(int alg, int W, const u64* gen, size_t lim, F f) {
  if (alg != 0) {
    for (size_t p = 0; p < lim; ++p) f(p);
    return;
  }
  for (int wi = 0; wi < W; ++wi) {
    u64 sup = (gen[wi] | (gen[wi] >> 1)) & EVEN;
    while (sup) {
      const size_t p = (size_t)wi * 64 + __builtin_ctzll(sup);
      sup &= sup - 1;
      if (p < lim) f(p);
      if (p + 1 < lim) f(p + 1);
    }
  }
}

// --------------------------------------------------------------- tableau
// A deferred Clifford frame (crates/core/src/algebra/tableau.rs:29-223):
// 2n rows, a readout map P -> C^dag P C and its inverse generator map.
struct Tableau {
  int alg = 0, W = 1;
  size_t rows = 0;
  std::vector<u64> rd_img, gen_img;  // rows x W
  std::vector<int> rd_sign, gen_sign;
  bool identity = true;

  Tableau() = default;
  Tableau(int a, int w, u32 n_units) : alg(a), W(w), rows(2 * (size_t)n_units) {
    rd_img.assign(rows * W, 0);
    rd_sign.assign(rows, 1);
    for (size_t p = 0; p < rows; ++p)
      if (p < (size_t)64 * W) rd_img[p * W + p / 64] = 1ULL << (p % 64);
    gen_img = rd_img;
    gen_sign = rd_sign;
  }
  bool row_is_unit(const std::vector<u64>& img, size_t p) const {
    for (int i = 0; i < W; ++i) {
      u64 want = (p < (size_t)64 * W && (size_t)i == p / 64) ? (1ULL << (p % 64)) : 0;
      if (img[p * W + i] != want) return false;
    }
    return true;
  }
  void refresh_identity() {
    identity = true;
    for (size_t p = 0; p < rows && identity; ++p)
      if (!row_is_unit(rd_img, p) || rd_sign[p] != 1) identity = false;
  }
  // apply_rows (tableau.rs:109-143) with phases as exponents of i: the image
  // of `mono` as the product of the images of its unit bits.
  int apply(const std::vector<u64>& img, const std::vector<int>& sgn, const u64* mono, u64* out) const {
    u64 src[MAX_WORDS] = {0}, e[MAX_WORDS] = {0};
    for (int i = 0; i < W; ++i) out[i] = 0;
    int se = 0, ie = 0;
    for (int wi = 0; wi < W; ++wi) {
      u64 bits = mono[wi];
      while (bits) {
        int b = __builtin_ctzll(bits);
        bits &= bits - 1;
        size_t p = (size_t)wi * 64 + b;
        if (p >= rows) continue;
        e[wi] = 1ULL << b;
        se += host_product_exp(alg, W, e, src);
        src[wi] ^= e[wi];
        e[wi] = 0;
        const u64* g = &img[p * W];
        ie += host_product_exp(alg, W, g, out) + (sgn[p] < 0 ? 2 : 0);
        for (int i = 0; i < W; ++i) out[i] ^= g[i];
      }
    }
    return (((ie - se) & 3) == 2) ? -1 : 1;
  }
  int conjugate_generator(const u64* mono, u64* out) const {
    if (identity) {
      std::memcpy(out, mono, 8 * W);
      return 1;
    }
    return apply(gen_img, gen_sign, mono, out);
  }
  // The frame followed by `next` (both maps), by full composition.
  void compose(const Tableau& next) {
    if (next.identity) return;
    std::vector<u64> r2(rows * W), g2(next.rows * W);
    std::vector<int> rs(rows), gs(next.rows);
    for (size_t i = 0; i < rows; ++i) rs[i] = next.apply(next.rd_img, next.rd_sign, &rd_img[i * W], &r2[i * W]) * rd_sign[i];
    for (size_t i = 0; i < next.rows; ++i)
      gs[i] = apply(gen_img, gen_sign, &next.gen_img[i * W], &g2[i * W]) * next.gen_sign[i];
    rd_img.swap(r2);
    rd_sign.swap(rs);
    gen_img.swap(g2);
    gen_sign.swap(gs);
    refresh_identity();
  }
  // for_rotation (tableau.rs:180-209), for |cos(angle)| < eps.
  static Tableau for_rotation(int alg, int W, u32 n_units, const u64* gen, double angle) {
    Tableau t(alg, W, n_units);
    const double sn = std::sin(angle);
    size_t lim = std::min(t.rows, (size_t)64 * W);
    u64 e[MAX_WORDS] = {0};
    for (size_t p = 0; p < lim; ++p) {
      e[p / 64] = 1ULL << (p % 64);
      const bool anti = host_anticommutes(alg, W, gen, e);
      const int pe = anti ? host_product_exp(alg, W, gen, e) : 0;
      e[p / 64] = 0;
      if (!anti) continue;
      const int s = rotated_sign(sn, pe);
      for (int i = 0; i < W; ++i) t.rd_img[p * W + i] = t.gen_img[p * W + i] = gen[i];
      t.rd_img[p * W + p / 64] ^= 1ULL << (p % 64);
      t.gen_img[p * W + p / 64] ^= 1ULL << (p % 64);
      t.rd_sign[p] = s;
      t.gen_sign[p] = -s;
    }
    t.refresh_identity();
    return t;
  }
  // compose(for_rotation(gen, angle)) without building the rotation's
  // tableau: O(rows x W) instead of O(rows x weight x W) per rotation.
  //   readout: each image that anticommutes with G becomes
  //     rotated_sign(sn, p) (G xor image), the conjugation of the image itself;
  //   generators: only the unit rows e_p that anticommute with G change, to
  //     the old generator map applied to -rotated_sign (G xor e_p).
  void compose_rotation(const u64* gen, double angle) {
    const double sn = std::sin(angle);
    for (size_t p = 0; p < rows; ++p) {
      u64* img = &rd_img[p * W];
      if (!host_anticommutes(alg, W, gen, img)) continue;
      rd_sign[p] *= rotated_sign(sn, host_product_exp(alg, W, gen, img));
      for (int i = 0; i < W; ++i) img[i] ^= gen[i];
    }
    const size_t lim = std::min(rows, (size_t)64 * W);
    std::vector<size_t> changed;
    std::vector<u64> imgs;
    std::vector<int> sgns;
    u64 e[MAX_WORDS] = {0}, m[MAX_WORDS];
    for_candidate_units(alg, W, gen, lim, [&](size_t p) {
      e[p / 64] = 1ULL << (p % 64);
      const bool anti = host_anticommutes(alg, W, gen, e);
      const int pe = anti ? host_product_exp(alg, W, gen, e) : 0;
      e[p / 64] = 0;
      if (!anti) return;
      for (int i = 0; i < W; ++i) m[i] = gen[i];
      m[p / 64] ^= 1ULL << (p % 64);
      changed.push_back(p);
      imgs.resize(imgs.size() + W);
      sgns.push_back(apply(gen_img, gen_sign, m, &imgs[imgs.size() - W]) * -rotated_sign(sn, pe));
    });
    for (size_t c = 0; c < changed.size(); ++c) {
      std::memcpy(&gen_img[changed[c] * W], &imgs[c * W], 8 * W);
      gen_sign[changed[c]] = sgns[c];
    }
    refresh_identity();
  }
  // changes_weight of for_rotation(gen) without building the tableau: a
  // single-bit row keeps its image unless it anticommutes with gen, and then
  // its image is gen ^ e_p.
  static bool rotation_changes_weight(int alg, int W, u32 n_units, const u64* gen) {
    const size_t lim = std::min((size_t)2 * n_units, (size_t)64 * W);
    u64 e[MAX_WORDS] = {0}, img[MAX_WORDS];
    bool changes = false;
    for_candidate_units(alg, W, gen, lim, [&](size_t p) {
      if (changes) return;
      e[p / 64] = 1ULL << (p % 64);
      const bool anti = host_anticommutes(alg, W, gen, e);
      e[p / 64] = 0;
      if (!anti) return;
      for (int i = 0; i < W; ++i) img[i] = gen[i];
      img[p / 64] ^= 1ULL << (p % 64);
      if (host_support(W, img) != 1) changes = true;
    });
    return changes;
  }
};

}  // namespace pqh
