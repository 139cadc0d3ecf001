// pq_oracle.cpp -- TEST INFRASTRUCTURE, not product code.
//
// A CPU restatement of propaq's numerical propagation engine, used as the
// checker for the CUDA engine and as the timed CPU baseline.  It follows the
// reference's algorithm step by step, with its own data structures:
//
//   * BasisString bit operations      crates/core/src/algebra/strings.rs:118-162
//   * Pauli algebra                   crates/pauli/src/algebra.rs:130-240
//   * Majorana algebra                crates/majorana/src/algebra.rs:32-216,
//                                     crates/majorana/src/monomial.rs:688-718
//   * f64 rotation arithmetic         crates/core/src/algebra/coeff.rs:115-209
//   * Clifford tableau (deferral)     crates/core/src/algebra/tableau.rs:38-223
//   * EmitCutoff / EmitPrecheck       crates/core/src/engine/termsum.rs:46-197
//   * per-partition TermSum           crates/core/src/engine/termsum.rs:208-862
//   * PartitionedTermSum              crates/core/src/engine/partitioned_termsum.rs:112-697
//   * run_at_width driver             crates/pauli/src/engine.rs:74-238
//   * noise resolution                crates/core/src/engine/noise_resolver.rs:51-131
//   * plugin loaders                  crates/core/src/policy/native_noise.rs,
//                                     crates/core/src/policy/native_truncator.rs
//
// Partitions are worker threads, as the reference's rayon partitions are.  The
// partition of a key is (hash >> 32) % S like termsum.rs:872-877, but with this
// file's own 64-bit hash rather than FxHash, so the row order inside a
// partition can differ from the reference's; the term set and every
// coefficient do not depend on it (the reference's own tests assert
// partition-count invariance, crates/core/tests/unit/engine/partitioned_termsum.rs).

#include "pq_oracle.h"

#include <dlfcn.h>

#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

using u64 = uint64_t;
using u32 = uint32_t;

constexpr u64 EVEN = 0x5555555555555555ULL;
constexpr double EPS_CLASSIFY = 1e-9;  // PHASE_ONLY_EPS, termsum.rs:42 / partitioned_termsum.rs:41
constexpr size_t KERNEL_BATCH = 1024;  // term_kernel.rs:93

thread_local std::string g_last_error;

inline int popc(u64 x) { return __builtin_popcountll(x); }

template <int W>
struct Key {
  u64 w[W];
  bool operator==(const Key& o) const {
    for (int i = 0; i < W; ++i)
      if (w[i] != o.w[i]) return false;
    return true;
  }
  bool operator!=(const Key& o) const { return !(*this == o); }
  static Key zero() {
    Key k;
    for (int i = 0; i < W; ++i) k.w[i] = 0;
    return k;
  }
  static Key unit(int p) {
    Key k = zero();
    if (p < 64 * W) k.w[p / 64] |= 1ULL << (p % 64);
    return k;
  }
  bool test(int p) const { return (w[p / 64] >> (p % 64)) & 1; }
  Key operator^(const Key& o) const {
    Key r;
    for (int i = 0; i < W; ++i) r.w[i] = w[i] ^ o.w[i];
    return r;
  }
  int count() const {
    int n = 0;
    for (int i = 0; i < W; ++i) n += popc(w[i]);
    return n;
  }
  int count_and(const Key& o) const {
    int n = 0;
    for (int i = 0; i < W; ++i) n += popc(w[i] & o.w[i]);
    return n;
  }
  bool parity_and(const Key& o) const {
    u64 acc = 0;
    for (int i = 0; i < W; ++i) acc ^= w[i] & o.w[i];
    return popc(acc) & 1;
  }
  // Units with either of their two bits set (strings.rs:140-148).
  int support() const {
    int n = 0;
    for (int i = 0; i < W; ++i) n += popc((w[i] | (w[i] >> 1)) & EVEN);
    return n;
  }
  // Swap the two bits of every unit pair (strings.rs:155-162).
  Key pair_swap() const {
    Key r;
    for (int i = 0; i < W; ++i) r.w[i] = ((w[i] & EVEN) << 1) | ((w[i] >> 1) & EVEN);
    return r;
  }
  template <class F>
  void for_each_position(F f) const {
    for (int i = 0; i < W; ++i) {
      u64 r = w[i];
      while (r) {
        int b = __builtin_ctzll(r);
        r &= r - 1;
        f(i * 64 + b);
      }
    }
  }
};

// Oracle's own key hash: a splitmix64 finaliser folded over the words.
inline u64 mix64(u64 x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
template <int W>
inline u64 key_hash(const Key<W>& k) {
  u64 h = mix64(k.w[0]);
  for (int i = 1; i < W; ++i) h = mix64(h ^ k.w[i]);
  return h;
}

// A unit complex phase, with num-complex's multiplication and division.
struct Phase {
  double re, im;
};
inline Phase pmul(Phase a, Phase b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline Phase pscale(Phase a, double s) { return {a.re * s, a.im * s}; }
inline Phase pdiv(Phase a, Phase b) {
  double n = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / n, (a.im * b.re - a.re * b.im) / n};
}
inline Phase i_pow(int p) {
  switch (p) {
    case 0: return {1.0, 0.0};
    case 1: return {0.0, 1.0};
    case 2: return {-1.0, 0.0};
    default: return {0.0, -1.0};
  }
}
inline int mod4(int v) { return ((v % 4) + 4) % 4; }

// ---------------------------------------------------------------- Pauli
// crates/pauli/src/algebra.rs: bit 2q = x of qubit q, bit 2q+1 = z of qubit q.
template <int W>
struct PauliAlg {
  static constexpr u32 KIND = 0;
  struct Ctx {
    Key<W> gen, fold;
    int gen_y;
    double sign;
  };
  static int count_y(const Key<W>& m) {
    int n = 0;
    for (int i = 0; i < W; ++i) n += popc(m.w[i] & (m.w[i] >> 1) & EVEN);
    return n;
  }
  static int count_z_and_x(const Key<W>& a, const Key<W>& b) {
    int n = 0;
    for (int i = 0; i < W; ++i) n += popc((a.w[i] >> 1) & b.w[i] & EVEN);
    return n;
  }
  static Ctx make_ctx(const Key<W>& g, double sign = 1.0) { return Ctx{g, g.pair_swap(), count_y(g), sign}; }
  static bool anticommutes(const Ctx& c, const Key<W>& k) { return k.parity_and(c.fold); }
  static Key<W> product(const Ctx& c, const Key<W>& k, Phase* ph) {
    Key<W> out = k ^ c.gen;
    int p = mod4(c.gen_y + count_y(k) - count_y(out) + 2 * count_z_and_x(c.gen, k));
    *ph = pscale(i_pow(p), c.sign);
    return out;
  }
  static int product_exp(const Ctx& c, const Key<W>& k, Key<W>* out) {
    *out = k ^ c.gen;
    return mod4(c.gen_y + count_y(k) - count_y(*out) + 2 * count_z_and_x(c.gen, k));
  }
  static u32 weight(const Key<W>& k, u32) { return (u32)k.support(); }
  static double trace(const Key<W>& k, u32, const u64* diag, size_t nd) {
    for (int i = 0; i < W; ++i)
      if (k.w[i] & EVEN) return 0.0;
    u32 parity = 0;
    k.for_each_position([&](int pos) {
      size_t unit = pos / 2;
      u64 word = unit / 64 < nd ? diag[unit / 64] : 0;
      parity ^= (u32)((word >> (unit % 64)) & 1);
    });
    return parity == 0 ? 1.0 : -1.0;
  }
};

// ------------------------------------------------------------- Majorana
// crates/majorana/src/algebra.rs: bit m = Majorana mode m; site k owns 2k, 2k+1.
inline u64 gather_even(u64 x) {
  x &= 0x5555555555555555ULL;
  x = (x | (x >> 1)) & 0x3333333333333333ULL;
  x = (x | (x >> 2)) & 0x0f0f0f0f0f0f0f0fULL;
  x = (x | (x >> 4)) & 0x00ff00ff00ff00ffULL;
  x = (x | (x >> 8)) & 0x0000ffff0000ffffULL;
  return (x | (x >> 16)) & 0x00000000ffffffffULL;
}
inline int hermiticity_exp(int len) { return (len % 4 == 0 || len % 4 == 1) ? 0 : 1; }

template <int W>
struct MajoranaAlg {
  static constexpr u32 KIND = 1;
  struct Ctx {
    Key<W> gen;
    int gen_len;
    bool odd;
    double sign;
  };
  static Ctx make_ctx(const Key<W>& g, double sign = 1.0) {
    int len = g.count();
    return Ctx{g, len, (len & 1) == 1, sign};
  }
  static bool anticommutes(const Ctx& c, const Key<W>& k) {
    int overlap = k.count_and(c.gen);
    int cross = c.odd ? k.count() : 0;
    return ((cross + overlap) & 1) == 1;
  }
  // monomial.rs:696-718: parity of the transpositions that sort b's modes past a's.
  static bool resorting_parity(const Key<W>& a, const Key<W>& b) {
    u64 total = 0;
    for (int i = 0; i < W; ++i) total += popc(a.w[i]);
    u64 running = 0, count = 0;
    for (int wi = 0; wi < W; ++wi) {
      u64 aw = a.w[wi];
      running += popc(aw);
      u64 above_higher = total - running;
      u64 bw = b.w[wi];
      while (bw) {
        int bi = __builtin_ctzll(bw);
        u64 above_same = bi < 63 ? (u64)popc(aw >> (bi + 1)) : 0;
        count += above_same + above_higher;
        bw &= bw - 1;
      }
    }
    return count & 1;
  }
  static int product_exp(const Ctx& c, const Key<W>& k, Key<W>* out) {
    *out = k ^ c.gen;
    int ra = hermiticity_exp(c.gen_len);
    int rb = hermiticity_exp(k.count());
    int rc = hermiticity_exp(out->count());
    int sw = resorting_parity(c.gen, k) ? 1 : 0;
    return mod4(ra + rb - rc + 2 * sw);
  }
  static Key<W> product(const Ctx& c, const Key<W>& k, Phase* ph) {
    Key<W> out;
    int p = product_exp(c, k, &out);
    *ph = pscale(i_pow(p), c.sign);
    return out;
  }
  // jw_weight, crates/majorana/src/algebra.rs:85-123.
  static u32 weight(const Key<W>& m, u32 n_sites) {
    if (n_sites == 0) return 0;
    u64 x[W], y[W];
    for (int i = 0; i < W; ++i) x[i] = y[i] = 0;
    for (int w = 0; w < W; ++w) {
      int half = 32 * (w % 2);
      x[w / 2] |= gather_even(m.w[w]) << half;
      y[w / 2] |= gather_even(m.w[w] >> 1) << half;
    }
    u64 single[W], occupied[W], p[W];
    for (int i = 0; i < W; ++i) {
      single[i] = x[i] ^ y[i];
      occupied[i] = x[i] | y[i];
      p[i] = single[i];
    }
    auto mask_to = [&](u64* v, size_t n) {
      for (int i = 0; i < W; ++i) {
        size_t low = (size_t)i * 64;
        u64 m2 = low >= n ? 0 : (n - low >= 64 ? ~0ULL : ((1ULL << (n - low)) - 1));
        v[i] &= m2;
      }
    };
    for (size_t shift = 1; shift < n_sites; shift <<= 1) {
      u64 src[W];
      for (int i = 0; i < W; ++i) src[i] = p[i];
      size_t words = shift / 64, bits = shift % 64;
      for (int i = W - 1; i >= (int)words; --i) {
        u64 v = src[i - words] << bits;
        if (bits > 0 && i > (int)words) v |= src[i - words - 1] >> (64 - bits);
        p[i] ^= v;
      }
      mask_to(p, n_sites);
    }
    int nsingle = 0;
    for (int i = 0; i < W; ++i) nsingle += popc(single[i]);
    bool odd_single = nsingle & 1;
    u32 weight = 0;
    for (int i = 0; i < W; ++i) {
      size_t low = (size_t)i * 64;
      u64 live = low >= n_sites ? 0 : (n_sites - low >= 64 ? ~0ULL : ((1ULL << (n_sites - low)) - 1));
      u64 str = odd_single ? (p[i] ^ live) : p[i];
      weight += popc(single[i] | (occupied[i] ^ str));
    }
    return weight;
  }
  static double trace(const Key<W>& k, u32 n_sites, const u64* diag, size_t nd) {
    int paired = 0, product = 1;
    for (u32 s = 0; s < n_sites; ++s) {
      bool lo = k.test(2 * s), hi = k.test(2 * s + 1);
      if (lo != hi) return 0.0;
      if (lo) {
        u64 word = s / 64 < nd ? diag[s / 64] : 0;
        int nk = (int)((word >> (s % 64)) & 1);
        product *= 2 * nk - 1;
        paired += 1;
      }
    }
    int phase = ((paired / 2) % 2 == 0) ? 1 : -1;
    return (double)(phase * product);
  }
};

// ------------------------------------------------------------- Tableau
// crates/core/src/algebra/tableau.rs
template <int W, class A>
struct Tableau {
  struct Row {
    Key<W> image;
    double sign;
  };
  std::vector<Row> readout, generator;
  bool identity = true;

  explicit Tableau(u32 n_units) {
    readout.resize(2 * (size_t)n_units);
    for (size_t p = 0; p < readout.size(); ++p) readout[p] = Row{Key<W>::unit((int)p), 1.0};
    generator = readout;
    identity = true;
  }
  void refresh_identity() {
    identity = true;
    for (size_t p = 0; p < readout.size(); ++p) {
      if (readout[p].image != Key<W>::unit((int)p) || readout[p].sign != 1.0) {
        identity = false;
        return;
      }
    }
  }
  static std::pair<Key<W>, double> apply_rows(const std::vector<Row>& rows, const Key<W>& mono) {
    Key<W> source = Key<W>::zero(), image = Key<W>::zero();
    Phase sp{1.0, 0.0}, ip{1.0, 0.0};
    mono.for_each_position([&](int p) {
      if ((size_t)p >= rows.size()) return;
      const Row& row = rows[p];
      Phase ph;
      source = A::product(A::make_ctx(Key<W>::unit(p)), source, &ph);
      sp = pmul(sp, ph);
      image = A::product(A::make_ctx(row.image), image, &ph);
      ip = pmul(ip, pscale(ph, row.sign));
    });
    Phase ratio = pdiv(ip, sp);
    return {image, ratio.re >= 0.0 ? 1.0 : -1.0};
  }
  std::pair<Key<W>, double> conjugate(const Key<W>& m) const {
    if (identity) return {m, 1.0};
    return apply_rows(readout, m);
  }
  std::pair<Key<W>, double> conjugate_generator(const Key<W>& m) const {
    if (identity) return {m, 1.0};
    return apply_rows(generator, m);
  }
  void compose(const Tableau& next) {
    if (next.identity) return;
    std::vector<Row> r2(readout.size()), g2(next.generator.size());
    for (size_t i = 0; i < readout.size(); ++i) {
      auto pr = apply_rows(next.readout, readout[i].image);
      r2[i] = Row{pr.first, pr.second * readout[i].sign};
    }
    for (size_t i = 0; i < next.generator.size(); ++i) {
      auto pr = apply_rows(generator, next.generator[i].image);
      g2[i] = Row{pr.first, pr.second * next.generator[i].sign};
    }
    readout = std::move(r2);
    generator = std::move(g2);
    refresh_identity();
  }
  // for_rotation: only when |cos(angle)| < eps.
  static bool for_rotation(u32 n_units, const Key<W>& gen, double angle, Tableau* out) {
    if (!(std::fabs(std::cos(angle)) < EPS_CLASSIFY)) return false;
    auto ctx = A::make_ctx(gen);
    Tableau t(n_units);
    size_t lim = std::min(t.readout.size(), (size_t)(64 * W));
    for (size_t p = 0; p < lim; ++p) {
      Key<W> g = Key<W>::unit((int)p);
      if (!A::anticommutes(ctx, g)) continue;
      Phase ph;
      Key<W> image = A::product(ctx, g, &ph);
      double sign = std::sin(angle) * (-ph.im);
      t.readout[p] = Row{image, sign};
      t.generator[p] = Row{image, -sign};
    }
    t.refresh_identity();
    *out = std::move(t);
    return true;
  }
  bool changes_weight() const {
    for (size_t p = 0; p < readout.size(); ++p)
      if (readout[p].image.support() != Key<W>::unit((int)p).support()) return true;
    return false;
  }
};

// ------------------------------------------------------------- plugins
struct Plugin {
  bool is_noise = true;
  void* lib = nullptr;
  void* ctx = nullptr;
  u32 depends = 0;
  void* fn = nullptr;        // factor / keep
  void* batch_fn = nullptr;  // factor_batch / keep_batch
  void (*destroy)(void*) = nullptr;
  ~Plugin() {
    if (destroy) destroy(ctx);
    if (lib) dlclose(lib);
  }
};
typedef double (*NoiseFactorFn)(void*, u32, const u64*, size_t, u32, u32, u32, u32);
typedef int32_t (*NoiseBatchFn)(void*, u32, const u64*, size_t, u32, const u32*, u32, u32, double*, size_t);
typedef int32_t (*KeepFn)(void*, u32, const u64*, size_t, u32, u32, double, u32, u32);
typedef int32_t (*KeepBatchFn)(void*, u32, const u64*, size_t, u32, const u32*, const double*, u32, u32,
                               uint8_t*, size_t);

int load_plugin(bool noise, const char* path, const char* config, void** out, char* err, size_t err_len) {
  const char* kind = noise ? "noise" : "truncator";
  const std::string pre = noise ? "propaq_noise_" : "propaq_truncator_";
  auto fail = [&](int code, const std::string& msg) {
    if (err && err_len) snprintf(err, err_len, "%s", msg.c_str());
    return code;
  };
  void* lib = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!lib) return fail(1, std::string("failed to load ") + kind + " plugin '" + path + "': " + dlerror());
  auto sym = [&](const char* name) { return dlsym(lib, (pre + name).c_str()); };
  auto abi = (u32(*)(void))sym("abi_version");
  if (!abi) {
    dlclose(lib);
    return fail(2, std::string(kind) + " plugin '" + path + "' does not export " + pre + "abi_version");
  }
  u32 ver = abi();
  if (ver != 1) {
    dlclose(lib);
    return fail(2, std::string(kind) + " plugin '" + path + "' targets ABI version " + std::to_string(ver) +
                       ", expected 1");
  }
  u32 dep = 0;
  if (auto d = (u32(*)(void))sym("depends")) {
    dep = d();
    if (dep & ~3u) {
      dlclose(lib);
      char buf[64];
      snprintf(buf, sizeof buf, "%#x", dep);
      return fail(2, std::string(kind) + " plugin '" + path + "' declares unknown dependency bits " + buf);
    }
  }
  void* fn = sym(noise ? "factor" : "keep");
  if (!fn) {
    dlclose(lib);
    return fail(2, std::string(kind) + " plugin '" + path + "' does not export " + pre + (noise ? "factor" : "keep"));
  }
  void* bfn = sym(noise ? "factor_batch" : "keep_batch");
  auto create = (void* (*)(const char*))sym("create");
  auto destroy = (void (*)(void*))sym("destroy");
  if ((create != nullptr) != (destroy != nullptr)) {
    dlclose(lib);
    return fail(2, std::string(kind) + " plugin '" + path + "' must export both " + pre + "create and " + pre +
                       "destroy, or neither");
  }
  auto* p = new Plugin();
  p->is_noise = noise;
  p->lib = lib;
  p->depends = dep;
  p->fn = fn;
  p->batch_fn = bfn;
  p->destroy = destroy;
  p->ctx = create ? create(config) : nullptr;
  *out = p;
  return 0;
}

// ------------------------------------------------------------- thread pool
class Pool {
 public:
  explicit Pool(int n) : n_(n) {
    for (int i = 1; i < n; ++i) threads_.emplace_back([this, i] { loop(i); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
      ++gen_;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
  }
  int size() const { return n_; }
  void run(const std::function<void(int)>& f) {
    if (n_ == 1) {
      f(0);
      return;
    }
    {
      std::lock_guard<std::mutex> g(m_);
      job_ = &f;
      pending_ = n_ - 1;
      ++gen_;
    }
    cv_.notify_all();
    f(0);
    std::unique_lock<std::mutex> g(m_);
    done_cv_.wait(g, [this] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  void loop(int idx) {
    u64 seen = 0;
    for (;;) {
      const std::function<void(int)>* job;
      {
        std::unique_lock<std::mutex> g(m_);
        cv_.wait(g, [&] { return gen_ != seen; });
        seen = gen_;
        if (stop_) return;
        job = job_;
      }
      (*job)(idx);
      {
        std::lock_guard<std::mutex> g(m_);
        if (--pending_ == 0) done_cv_.notify_one();
      }
    }
  }
  int n_;
  std::vector<std::thread> threads_;
  std::mutex m_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)>* job_ = nullptr;
  int pending_ = 0;
  u64 gen_ = 0;
  bool stop_ = false;
};

// ------------------------------------------------------------- cutoff
struct Cutoff {
  bool has_w = false;
  u32 max_weight = 0;
  bool has_c = false;
  double min_coeff = 0;
  Plugin* term = nullptr;
  bool has_floor = false;
  u64 min_terms = 0;
  u32 layer = 0, n_layers = 0;
  Cutoff lossless() const {
    Cutoff c;
    c.has_floor = has_floor;
    c.min_terms = min_terms;
    c.layer = layer;
    c.n_layers = n_layers;
    return c;
  }
  Cutoff at_size(u64 n_live) const { return (has_floor && n_live < min_terms) ? lossless() : *this; }
};

template <int W, class A>
struct Routed {
  Key<W> key;
  u64 hash;
  double coeff;
};

// Open-addressing index: slot = (row, folded hash), linear probing, load <= 0.7
// (the reference's OperatorIndex layout, operator_index.rs:129-475).
template <int W>
struct Index {
  std::vector<u64> slots;  // hi 32 = fp, lo 32 = row; ~0 empty
  u64 mask = 0;
  size_t used = 0;
  void reset(size_t expect) {
    size_t cap = 16;
    while (cap * 7 < expect * 10 + 10) cap <<= 1;
    slots.assign(cap, ~0ULL);
    mask = cap - 1;
    used = 0;
  }
  template <class KeysVec>
  long find(const Key<W>& k, u64 h, const KeysVec& keys) const {
    u64 i = (h ^ (h >> 29)) & mask;
    u32 fp = (u32)(h >> 32);
    for (;;) {
      u64 s = slots[i];
      if (s == ~0ULL) return -1;
      if ((u32)(s >> 32) == fp && keys[(u32)s] == k) return (long)(u32)s;
      i = (i + 1) & mask;
    }
  }
  template <class KeysVec>
  void insert(u32 row, u64 h, const KeysVec& keys) {
    if ((used + 1) * 10 > slots.size() * 7) grow(keys);
    u64 i = (h ^ (h >> 29)) & mask;
    while (slots[i] != ~0ULL) i = (i + 1) & mask;
    slots[i] = ((h >> 32) << 32) | row;
    ++used;
  }
  template <class KeysVec>
  void grow(const KeysVec& keys) {
    std::vector<u64> old = std::move(slots);
    slots.assign(old.size() * 2, ~0ULL);
    mask = slots.size() - 1;
    for (u64 s : old) {
      if (s == ~0ULL) continue;
      u64 h = key_hash<W>(keys[(u32)s]);
      u64 i = (h ^ (h >> 29)) & mask;
      while (slots[i] != ~0ULL) i = (i + 1) & mask;
      slots[i] = s;
    }
  }
};

// ------------------------------------------------------------- TermSum
// One hash partition, crates/core/src/engine/termsum.rs:208-862.
template <int W, class A>
struct TermSum {
  using K = Key<W>;
  using Ctx = typename A::Ctx;
  u32 n_units;
  std::vector<K> keys;
  std::vector<double> coeffs;
  Index<W> index;
  std::vector<u32> pending_slot, pending_rows, claimed_rows;
  std::vector<double> pending_vals;
  bool pending_needs_phase = false;
  u64 emitted = 0, hits = 0, visited = 0, declined = 0;
  double discarded_l1 = 0, discarded_max = 0;

  explicit TermSum(u32 n) : n_units(n) { index.reset(16); }
  size_t len() const { return keys.size(); }

  void add(const K& k, double c) {
    u64 h = key_hash<W>(k);
    long r = index.find(k, h, keys);
    if (r >= 0) {
      coeffs[r] += c;
      return;
    }
    push(k, h, c);
  }
  void push(const K& k, u64 h, double c) {
    u32 row = (u32)keys.size();
    keys.push_back(k);
    coeffs.push_back(c);
    index.insert(row, h, keys);
  }

  // admits_key / admits_child / admits_initial / admits_coeff (termsum.rs:113-168).
  bool admits_key(const Cutoff& c, const K& k) const {
    if (c.term) return true;
    return !c.has_w || A::weight(k, n_units) <= c.max_weight;
  }
  bool admits_child(const Cutoff& c, const K& k, double coeff) const {
    if (c.term) {
      auto keep = (KeepFn)c.term->fn;
      bool key_dep = c.term->depends & 1;
      return keep(c.term->ctx, A::KIND, key_dep ? k.w : nullptr, key_dep ? (size_t)W : 0, n_units,
                  A::weight(k, n_units), std::fabs(coeff), c.layer, c.n_layers) != 0;
    }
    return !c.has_c || std::fabs(coeff) >= c.min_coeff;
  }
  bool admits_initial(const Cutoff& c, const K& k, double coeff) const {
    return admits_key(c, k) && admits_child(c, k, coeff);
  }

  void scale_by_table(const double* table, size_t len) {
    for (size_t i = 0; i < keys.size(); ++i) {
      u32 w = A::weight(keys[i], n_units);
      coeffs[i] *= table[std::min<size_t>(w, len - 1)];
    }
  }
  // scale_by_key, termsum.rs:340-371.
  void scale_by_key(Plugin* p, u32 layer, u32 n_layers) {
    size_t n = keys.size();
    if (n == 0) return;
    size_t chunk = std::min(KERNEL_BATCH, n);
    std::vector<u64> words(chunk * W);
    std::vector<u32> weights(chunk);
    std::vector<double> factors(chunk);
    bool key_dep = p->depends & 1;
    for (size_t start = 0; start < n; start += chunk) {
      size_t len = std::min(chunk, n - start);
      for (size_t j = 0; j < len; ++j) {
        std::memcpy(&words[j * W], keys[start + j].w, sizeof(u64) * W);
        weights[j] = A::weight(keys[start + j], n_units);
      }
      bool done = false;
      if (p->batch_fn) {
        int rc = ((NoiseBatchFn)p->batch_fn)(p->ctx, A::KIND, key_dep ? words.data() : nullptr,
                                             key_dep ? (size_t)W : 0, n_units, weights.data(), layer, n_layers,
                                             factors.data(), len);
        done = rc == 0;
      }
      if (!done)
        for (size_t j = 0; j < len; ++j)
          factors[j] = ((NoiseFactorFn)p->fn)(p->ctx, A::KIND, key_dep ? &words[j * W] : nullptr,
                                              key_dep ? (size_t)W : 0, n_units, weights[j], layer, n_layers);
      for (size_t j = 0; j < len; ++j) coeffs[start + j] *= factors[j];
    }
  }

  template <class Keep>
  size_t reclaim(Keep keep) {
    size_t before = keys.size();
    std::vector<K> nk;
    std::vector<double> nc;
    nk.reserve(before);
    nc.reserve(before);
    Index<W> ni;
    ni.reset(before);
    for (size_t i = 0; i < before; ++i) {
      if (!keep(i)) continue;
      u32 row = (u32)nk.size();
      nk.push_back(keys[i]);
      nc.push_back(coeffs[i]);
      ni.insert(row, key_hash<W>(keys[i]), nk);
    }
    keys = std::move(nk);
    coeffs = std::move(nc);
    index = std::move(ni);
    pending_slot.clear();
    pending_rows.clear();
    pending_vals.clear();
    claimed_rows.clear();
    return before - keys.size();
  }
  size_t reclaim_cutoff(const Cutoff& c) {
    if (c.term) {
      // reclaim_by_kernel, termsum.rs:387-447
      size_t n = keys.size();
      std::vector<uint8_t> flags(n);
      size_t chunk = std::min(KERNEL_BATCH, std::max<size_t>(n, 1));
      std::vector<u64> words(chunk * W);
      std::vector<u32> weights(chunk);
      std::vector<double> mags(chunk);
      std::vector<uint8_t> dec(chunk);
      bool key_dep = c.term->depends & 1;
      for (size_t start = 0; start < n; start += chunk) {
        size_t len = std::min(chunk, n - start);
        for (size_t j = 0; j < len; ++j) {
          std::memcpy(&words[j * W], keys[start + j].w, sizeof(u64) * W);
          weights[j] = A::weight(keys[start + j], n_units);
          mags[j] = std::fabs(coeffs[start + j]);
        }
        bool batched = false;
        if (c.term->batch_fn) {
          batched = ((KeepBatchFn)c.term->batch_fn)(c.term->ctx, A::KIND, key_dep ? words.data() : nullptr,
                                                    key_dep ? (size_t)W : 0, n_units, weights.data(),
                                                    mags.data(), c.layer, c.n_layers, dec.data(), len) == 0;
        }
        for (size_t j = 0; j < len; ++j) {
          if (batched)
            flags[start + j] = dec[j] != 0;
          else
            flags[start + j] = ((KeepFn)c.term->fn)(c.term->ctx, A::KIND, key_dep ? &words[j * W] : nullptr,
                                                    key_dep ? (size_t)W : 0, n_units, weights[j], mags[j],
                                                    c.layer, c.n_layers) != 0;
        }
      }
      return reclaim([&](size_t i) { return flags[i] != 0; });
    }
    return reclaim([&](size_t i) { return admits_initial(c, keys[i], coeffs[i]); });
  }

  void scale_anticommuting(const Ctx& ctx, double f) {
    for (size_t i = 0; i < keys.size(); ++i)
      if (A::anticommutes(ctx, keys[i])) coeffs[i] *= f;
  }

  void reset_pending() {
    for (u32 r : pending_rows) pending_slot[r] = UINT32_MAX;
    pending_rows.clear();
    pending_vals.clear();
    claimed_rows.clear();
    if (pending_slot.size() < keys.size()) pending_slot.resize(keys.size(), UINT32_MAX);
  }
  void hold_back(size_t row, double c) {
    if (row >= pending_slot.size()) return;
    pending_slot[row] = (u32)pending_rows.size();
    pending_rows.push_back((u32)row);
    pending_vals.push_back(c);
  }
  void claim(size_t row) {
    if (row < pending_slot.size() && pending_slot[row] != UINT32_MAX) claimed_rows.push_back((u32)row);
  }

  // scan_into + emit_from_row, termsum.rs:561-601, 701-751.
  void scan_into(const Ctx& ctx, double sn, double cs, const Cutoff& cut, size_t S,
                 std::vector<std::vector<Routed<W, A>>>& outbox) {
    reset_pending();
    bool precheck = !cut.term && cut.has_c;
    pending_needs_phase = precheck;
    size_t n = keys.size();
    for (size_t i = 0; i < n; ++i) {
      if (!A::anticommutes(ctx, keys[i])) continue;
      ++visited;
      if (precheck && std::fabs(coeffs[i] * sn) < cut.min_coeff) {
        ++declined;
        hold_back(i, coeffs[i] * sn);
        coeffs[i] *= cs;
        continue;
      }
      Phase ph;
      K child = A::product(ctx, keys[i], &ph);
      double sin_branch = coeffs[i] * sn * (-ph.im);
      coeffs[i] *= cs;
      if (!admits_key(cut, child)) continue;
      if (!admits_child(cut, child, sin_branch)) {
        hold_back(i, sin_branch);
        ++declined;
        continue;
      }
      u64 h = key_hash<W>(child);
      ++emitted;
      outbox[S <= 1 ? 0 : (h >> 32) % S].push_back(Routed<W, A>{child, h, sin_branch});
    }
  }
  // absorb_routed, termsum.rs:788-800.
  bool absorb_routed(const Routed<W, A>& m) {
    long r = index.find(m.key, m.hash, keys);
    if (r >= 0) {
      ++hits;
      coeffs[r] += m.coeff;
      claim((size_t)r);
      return false;
    }
    push(m.key, m.hash, m.coeff);
    return true;
  }
  // drain_claims, termsum.rs:604-647.
  void drain_claims(const Ctx& ctx, size_t S, std::vector<std::vector<Routed<W, A>>>& outbox) {
    std::vector<u32> claims;
    claims.swap(claimed_rows);
    discarded_max = 0;
    if (claims.size() != pending_rows.size()) {
      std::vector<uint8_t> is_claimed(keys.size(), 0);
      for (u32 r : claims) is_claimed[r] = 1;
      for (size_t k = 0; k < pending_rows.size(); ++k) {
        if (!is_claimed[pending_rows[k]]) {
          double mag = std::fabs(pending_vals[k]);
          discarded_l1 += mag;
          if (mag > discarded_max) discarded_max = mag;
        }
      }
    }
    for (u32 row : claims) {
      u32 slot = pending_slot[row];
      Phase ph;
      K child = A::product(ctx, keys[row], &ph);
      u64 h = key_hash<W>(child);
      double c = pending_vals[slot];
      if (pending_needs_phase) c *= -ph.im;
      ++emitted;
      outbox[S <= 1 ? 0 : (h >> 32) % S].push_back(Routed<W, A>{child, h, c});
    }
  }
};

// ---------------------------------------------------------- partitioned
template <int W, class A>
struct Engine {
  using K = Key<W>;
  using TS = TermSum<W, A>;
  using Box = std::vector<std::vector<Routed<W, A>>>;
  u32 n_units;
  std::vector<TS> parts;
  Tableau<W, A> frame;
  bool defer_cliffords = true;
  Pool* pool;
  std::vector<Box> outboxes, rescues;

  Engine(u32 n, size_t S, Pool* p) : n_units(n), frame(n), pool(p) {
    for (size_t i = 0; i < S; ++i) parts.emplace_back(n);
    outboxes.assign(S, Box(S));
    rescues.assign(S, Box(S));
  }
  size_t S() const { return parts.size(); }
  size_t len() const {
    size_t n = 0;
    for (auto& p : parts) n += p.len();
    return n;
  }
  void add(const K& k, double c) {
    size_t S_ = S();
    size_t owner = S_ <= 1 ? 0 : (key_hash<W>(k) >> 32) % S_;
    parts[owner].add(k, c);
  }
  void par(const std::function<void(int)>& f) {
    if (S() == 1) {
      f(0);
      return;
    }
    pool->run(f);
  }
  size_t absorb_exchange(std::vector<Box>& boxes, const typename A::Ctx* ctx, std::vector<Box>* drain) {
    std::vector<size_t> added(S(), 0);
    size_t S_ = S();
    par([&](int dst) {
      for (size_t src = 0; src < S_; ++src)
        for (auto& m : boxes[src][dst])
          if (parts[dst].absorb_routed(m)) ++added[dst];
      if (drain) {
        for (auto& b : (*drain)[dst]) b.clear();
        parts[dst].drain_claims(*ctx, S_, (*drain)[dst]);
      }
    });
    size_t t = 0;
    for (size_t a : added) t += a;
    return t;
  }
  // apply_rotation, partitioned_termsum.rs:276-350.
  void apply_rotation(const K& gen_raw, double angle, const Cutoff& cutoff0) {
    if (len() == 0) return;
    Cutoff cut = cutoff0.at_size(len());
    if (defer_cliffords) {
      Tableau<W, A> step(0);
      if (Tableau<W, A>::for_rotation(n_units, gen_raw, angle, &step)) {
        if (!cut.has_w || !step.changes_weight()) {
          frame.compose(step);
          return;
        }
      }
    }
    auto gs = frame.conjugate_generator(gen_raw);
    auto ctx = A::make_ctx(gs.first, gs.second);
    double sn = std::sin(angle), cs = std::cos(angle);
    if (std::fabs(sn) < EPS_CLASSIFY) {
      par([&](int i) { parts[i].scale_anticommuting(ctx, cs); });
      return;
    }
    size_t S_ = S();
    par([&](int i) {
      for (auto& b : outboxes[i]) b.clear();
      parts[i].scan_into(ctx, sn, cs, cut, S_, outboxes[i]);
    });
    absorb_exchange(outboxes, &ctx, &rescues);
    bool any = false;
    for (auto& r : rescues)
      for (auto& b : r) any |= !b.empty();
    if (any) absorb_exchange(rescues, nullptr, nullptr);
  }
};

struct RunOut {
  std::vector<u64> keys;
  std::vector<double> coeffs;
  u32 n_words = 1;
};

template <int W, class A>
RunOut* run_impl(const pqo_config* cfg, const u64* obs_words, const double* obs_coeffs, size_t n_obs,
                 const u64* gate_words, const double* angles, size_t n_gates, const u32* layer_off,
                 size_t n_layers, const u64* diag, size_t nd, u64* n_terms_out, pqo_result* res) {
  using K = Key<W>;
  size_t S = cfg->n_partitions ? cfg->n_partitions : 1;
  std::unique_ptr<Pool> pool(S > 1 ? new Pool((int)S) : nullptr);
  Engine<W, A> op(cfg->n_units, S, pool.get());
  Cutoff cut;
  cut.has_w = cfg->max_weight >= 0;
  cut.max_weight = cut.has_w ? (u32)cfg->max_weight : 0;
  cut.has_c = cfg->has_min_coeff != 0;
  cut.min_coeff = cfg->min_coeff;
  cut.term = (Plugin*)cfg->truncator;
  cut.has_floor = cfg->min_terms >= 0;
  cut.min_terms = cut.has_floor ? (u64)cfg->min_terms : 0;

  Plugin* np = cfg->noise_kind == PQO_NOISE_PLUGIN ? (Plugin*)cfg->noise_plugin : nullptr;
  bool noise_key = np && (np->depends & 1);
  bool trunc_key = cut.term && (cut.term->depends & 1);
  if (trunc_key || noise_key) op.defer_cliffords = false;  // engine.rs:101-103

  // Noise resolution (noise_resolver.rs:78-131) for the plugin kind.
  std::vector<double> table;
  const u32 tlen = cfg->n_units + 1;
  auto retab = [&](u32 layer, u32 total) {
    table.resize(tlen);
    for (u32 w = 0; w < tlen; ++w)
      table[w] = ((NoiseFactorFn)np->fn)(np->ctx, A::KIND, nullptr, 0, cfg->n_units, w, layer, total);
  };
  if (np && !(np->depends & 1) && !(np->depends & 2)) retab(0, 0);

  for (size_t i = 0; i < n_obs; ++i) {
    K k;
    std::memcpy(k.w, obs_words + i * W, sizeof(u64) * W);
    if (!op.parts[0].admits_initial(cut, k, obs_coeffs[i])) continue;
    op.add(k, obs_coeffs[i]);
  }

  size_t g = 0;
  for (size_t l = 0; l < n_layers; ++l) {
    cut.layer = (u32)l;
    cut.n_layers = (u32)n_layers;
    if (cfg->noise_kind != PQO_NOISE_NONE) {
      if (cfg->noise_kind == PQO_NOISE_TABLE) {
        op.par([&](int i) { op.parts[i].scale_by_table(cfg->noise_tables, cfg->noise_table_len); });
      } else if (cfg->noise_kind == PQO_NOISE_LAYERED) {
        const double* t = cfg->noise_tables + l * cfg->noise_table_len;
        op.par([&](int i) { op.parts[i].scale_by_table(t, cfg->noise_table_len); });
      } else if (np) {
        if (np->depends & 1) {
          op.par([&](int i) { op.parts[i].scale_by_key(np, (u32)l, (u32)n_layers); });
        } else {
          if (np->depends & 2) retab((u32)l, (u32)n_layers);
          op.par([&](int i) { op.parts[i].scale_by_table(table.data(), table.size()); });
        }
      }
      if (cut.has_w || cut.has_c || cut.term)  // partitioned_termsum.rs:585-587
        op.par([&](int i) { op.parts[i].reclaim_cutoff(cut); });
    }
    for (u32 gi = layer_off[l]; gi < layer_off[l + 1]; ++gi, ++g) {
      K gen;
      std::memcpy(gen.w, gate_words + (size_t)gi * W, sizeof(u64) * W);
      op.apply_rotation(gen, angles[gi], cut);
      if (n_terms_out) n_terms_out[gi] = op.len();
    }
  }

  // Results (engine.rs:214-236, partitioned_termsum.rs:611-697).
  res->n_final = op.len();
  res->terms_below_cutoff = 0;
  if (cut.has_c)
    for (auto& p : op.parts)
      for (double c : p.coeffs) res->terms_below_cutoff += std::fabs(c) < cut.min_coeff;
  res->expectation = res->expectation_accurate = res->expectation_abs = 0;
  if (diag) {
    double total = 0, acc = 0, comp = 0, absum = 0;
    for (auto& p : op.parts) {
      double part = 0;
      for (size_t i = 0; i < p.len(); ++i) {
        double v;
        if (op.frame.identity) {
          v = p.coeffs[i] * A::trace(p.keys[i], cfg->n_units, diag, nd);
        } else {
          auto im = op.frame.conjugate(p.keys[i]);
          v = p.coeffs[i] * im.second * A::trace(im.first, cfg->n_units, diag, nd);
        }
        part += v;
        absum += std::fabs(v);
        double t = acc + v;
        comp += std::fabs(acc) >= std::fabs(v) ? (acc - t) + v : (v - t) + acc;
        acc = t;
      }
      total += part;
    }
    res->expectation = total;
    res->expectation_accurate = acc + comp;
    res->expectation_abs = absum;
  }
  res->emitted = res->hits = res->visited = res->declined = 0;
  res->discarded_l1 = 0;
  for (auto& p : op.parts) {
    res->emitted += p.emitted;
    res->hits += p.hits;
    res->visited += p.visited;
    res->declined += p.declined;
    res->discarded_l1 += p.discarded_l1;
  }
  auto* out = new RunOut();
  out->n_words = W;
  out->keys.reserve(op.len() * W);
  out->coeffs.reserve(op.len());
  for (auto& p : op.parts)
    for (size_t i = 0; i < p.len(); ++i) {
      auto im = op.frame.conjugate(p.keys[i]);
      for (int w = 0; w < W; ++w) out->keys.push_back(im.first.w[w]);
      out->coeffs.push_back(p.coeffs[i] * im.second);
    }
  return out;
}

template <int W>
RunOut* dispatch_alg(const pqo_config* c, const u64* ow, const double* oc, size_t no, const u64* gw,
                     const double* ga, size_t ng, const u32* lo, size_t nl, const u64* d, size_t nd, u64* nt,
                     pqo_result* r) {
  if (c->basis_kind == 0) return run_impl<W, PauliAlg<W>>(c, ow, oc, no, gw, ga, ng, lo, nl, d, nd, nt, r);
  return run_impl<W, MajoranaAlg<W>>(c, ow, oc, no, gw, ga, ng, lo, nl, d, nd, nt, r);
}

template <int W, class F>
auto with_key(const u64* src, F f) {
  Key<W> k;
  std::memcpy(k.w, src, sizeof(u64) * W);
  return f(k);
}

#define PQO_WIDTHS(X) X(1) X(2) X(4) X(8) X(16) X(32) X(64)

}  // namespace

extern "C" {

int pqo_load_noise(const char* path, const char* cfg, void** out, char* err, size_t n) {
  return load_plugin(true, path, cfg, out, err, n);
}
int pqo_load_truncator(const char* path, const char* cfg, void** out, char* err, size_t n) {
  return load_plugin(false, path, cfg, out, err, n);
}
void pqo_plugin_free(void* p) { delete (Plugin*)p; }
uint32_t pqo_plugin_depends(const void* p) { return ((const Plugin*)p)->depends; }

void* pqo_run(const pqo_config* cfg, const uint64_t* ow, const double* oc, size_t no, const uint64_t* gw,
              const double* ga, size_t ng, const uint32_t* lo, size_t nl, const uint64_t* d, size_t nd,
              uint64_t* nt, pqo_result* r) {
  try {
    std::memset(r, 0, sizeof(*r));
    switch (cfg->n_words) {
#define CASE(Wv) \
  case Wv:       \
    return dispatch_alg<Wv>(cfg, ow, oc, no, gw, ga, ng, lo, nl, d, nd, nt, r);
      PQO_WIDTHS(CASE)
#undef CASE
      default:
        g_last_error = "unsupported key width";
        return nullptr;
    }
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return nullptr;
  }
}
size_t pqo_terms_count(const void* run) { return ((const RunOut*)run)->coeffs.size(); }
void pqo_terms_copy(const void* run, uint64_t* keys, double* coeffs) {
  auto* r = (const RunOut*)run;
  std::memcpy(keys, r->keys.data(), r->keys.size() * sizeof(u64));
  std::memcpy(coeffs, r->coeffs.data(), r->coeffs.size() * sizeof(double));
}
void pqo_run_free(void* run) { delete (RunOut*)run; }
const char* pqo_last_error(void) { return g_last_error.c_str(); }

uint32_t pqo_weight(uint32_t kind, uint32_t n_units, uint32_t nw, const uint64_t* key) {
  switch (nw) {
#define CASE(Wv)                                                                   \
  case Wv:                                                                         \
    return with_key<Wv>(key, [&](const Key<Wv>& k) {                               \
      return kind == 0 ? PauliAlg<Wv>::weight(k, n_units) : MajoranaAlg<Wv>::weight(k, n_units); \
    });
    PQO_WIDTHS(CASE)
#undef CASE
  }
  return 0;
}
int pqo_anticommutes(uint32_t kind, uint32_t nw, const uint64_t* gen, const uint64_t* key) {
  switch (nw) {
#define CASE(Wv)                                                                          \
  case Wv: {                                                                              \
    Key<Wv> g, k;                                                                         \
    std::memcpy(g.w, gen, 8 * Wv);                                                        \
    std::memcpy(k.w, key, 8 * Wv);                                                        \
    return kind == 0 ? PauliAlg<Wv>::anticommutes(PauliAlg<Wv>::make_ctx(g), k)           \
                     : MajoranaAlg<Wv>::anticommutes(MajoranaAlg<Wv>::make_ctx(g), k);    \
  }
    PQO_WIDTHS(CASE)
#undef CASE
  }
  return 0;
}
int pqo_product(uint32_t kind, uint32_t nw, const uint64_t* gen, const uint64_t* key, uint64_t* child) {
  switch (nw) {
#define CASE(Wv)                                                                              \
  case Wv: {                                                                                  \
    Key<Wv> g, k, o;                                                                          \
    std::memcpy(g.w, gen, 8 * Wv);                                                            \
    std::memcpy(k.w, key, 8 * Wv);                                                            \
    int p = kind == 0 ? PauliAlg<Wv>::product_exp(PauliAlg<Wv>::make_ctx(g), k, &o)           \
                      : MajoranaAlg<Wv>::product_exp(MajoranaAlg<Wv>::make_ctx(g), k, &o);    \
    std::memcpy(child, o.w, 8 * Wv);                                                          \
    return p;                                                                                 \
  }
    PQO_WIDTHS(CASE)
#undef CASE
  }
  return -1;
}
double pqo_trace(uint32_t kind, uint32_t n_units, uint32_t nw, const uint64_t* key, const uint64_t* diag,
                 size_t nd) {
  switch (nw) {
#define CASE(Wv)                                                                               \
  case Wv:                                                                                     \
    return with_key<Wv>(key, [&](const Key<Wv>& k) {                                           \
      return kind == 0 ? PauliAlg<Wv>::trace(k, n_units, diag, nd)                            \
                       : MajoranaAlg<Wv>::trace(k, n_units, diag, nd);                        \
    });
    PQO_WIDTHS(CASE)
#undef CASE
  }
  return 0;
}

}  // extern "C"
