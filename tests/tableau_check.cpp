// Checks the deferred Clifford frame's direct rotation update
// (Tableau::compose_rotation) against full composition with the rotation's
// tableau (Tableau::compose(Tableau::for_rotation(...))), and
// Tableau::rotation_changes_weight against the rotation's full tableau, on
// random Clifford sequences, Pauli and Majorana, 1 and 2 key words: both maps, every row,
// every sign, and the conjugated generators of random rotations after each
// step.  Built and run by test_tableau_cpu.py; prints "ok" or the first
// difference.
#include <cstdio>
#include <random>

#include "../propaq_b200/csrc/pq_tableau.h"

using namespace pqh;

static void random_key(std::mt19937_64& rng, int alg, int W, u32 n_units, int max_units, u64* k) {
  for (int i = 0; i < W; ++i) k[i] = 0;
  const int n = 1 + (int)(rng() % (u64)max_units);
  for (int j = 0; j < n; ++j) {
    const u32 q = (u32)(rng() % n_units);
    const u64 bits = alg == 0 ? 1 + rng() % 3 : 1 + rng() % 3;  // X, Z, Y (or one or both modes)
    k[(2 * q) / 64] |= bits << ((2 * q) % 64);
  }
}

static bool same(const Tableau& a, const Tableau& b) {
  return a.rd_img == b.rd_img && a.gen_img == b.gen_img && a.rd_sign == b.rd_sign && a.gen_sign == b.gen_sign &&
         a.identity == b.identity;
}

int main() {
  std::mt19937_64 rng(12345);
  int cases = 0;
  for (int alg = 0; alg < 2; ++alg)
    for (int W : {1, 2})
      for (u32 n_units : {3u, 7u, (u32)(32 * W - 3), (u32)(32 * W)}) {
        if (n_units > 32u * W) continue;
        for (int seq = 0; seq < 6; ++seq) {
          Tableau fast(alg, W, n_units), full(alg, W, n_units);
          for (int step = 0; step < 40; ++step) {
            u64 g[MAX_WORDS];
            random_key(rng, alg, W, n_units, step % 5 == 4 ? (int)n_units : 3, g);
            const double ang = (rng() & 1) ? M_PI / 2 : -M_PI / 2;
            const Tableau rt = Tableau::for_rotation(alg, W, n_units, g, ang);
            bool want = false;  // a unit row whose image has another support
            for (size_t p = 0; p < rt.rows; ++p) {
              u64 u[MAX_WORDS] = {0};
              if (p < (size_t)64 * W) u[p / 64] = 1ULL << (p % 64);
              if (host_support(W, &rt.rd_img[p * W]) != host_support(W, u)) want = true;
            }
            if (Tableau::rotation_changes_weight(alg, W, n_units, g) != want) {
              std::printf("weight change differs: alg %d W %d n %u seq %d step %d\n", alg, W, n_units, seq, step);
              return 1;
            }
            fast.compose_rotation(g, ang);
            full.compose(rt);
            ++cases;
            if (!same(fast, full)) {
              std::printf("frame differs: alg %d W %d n %u seq %d step %d\n", alg, W, n_units, seq, step);
              return 1;
            }
            for (int t = 0; t < 4; ++t) {
              u64 h[MAX_WORDS], o1[MAX_WORDS], o2[MAX_WORDS];
              random_key(rng, alg, W, n_units, 4, h);
              const int s1 = fast.conjugate_generator(h, o1), s2 = full.conjugate_generator(h, o2);
              if (s1 != s2 || std::memcmp(o1, o2, 8 * W) != 0) {
                std::printf("conjugated generator differs: alg %d W %d n %u\n", alg, W, n_units);
                return 1;
              }
            }
          }
        }
      }
  std::printf("ok %d\n", cases);
  return 0;
}
