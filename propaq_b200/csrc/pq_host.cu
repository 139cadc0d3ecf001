// pq_host.cu -- host side of the B200 propagation engine and its C ABI.
//
// The host owns the control flow the reference runs in
// crates/pauli/src/engine.rs:74-238 (run_at_width) and
// crates/core/src/engine/partitioned_termsum.rs:276-350 (apply_rotation):
//   * observable admission and duplicate folding (engine.rs:104-111);
//   * per layer: the noise op (a damping + reclaim kernel) at the start of the
//     layer, then one op per gate (engine.rs:117-205);
//   * per gate: TermBudget floor, Clifford deferral into a host-side tableau,
//     generator conjugation through it, phase-only classification, then the
//     branch kernel (partitioned_termsum.rs:282-350);
//   * the expectation value and the final terms through the readout frame.
// sin/cos/exp are evaluated here with the host libm, the same glibc the
// reference calls, so the device sees bit-identical factors.
//
// Ops are enqueued without waiting for the device.  Each gate kernel first
// checks that twice the live count fits the row capacity; if not, it and every
// later op skip themselves and record where they stopped.  The host notices at
// its next synchronisation, grows the buffers, rebuilds the hash table and
// replays the ops from the one that stopped.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/propaq_cuda.h"
#include "pq_kernels.cuh"

using pq::u32;
using pq::u64;

namespace {

constexpr double EPS_CLASSIFY = 1e-9;  // termsum.rs:42, partitioned_termsum.rs:41
constexpr u32 MAX_UNITS = 2048;        // engine.rs:27
constexpr u64 MAX_ROWS = 1ULL << 31;   // row index ceiling of the table slots
constexpr int TILE_ROWS = 256;  // smallest tile a sweep uses (sizes the look-back status array)

inline int hpopc(u64 x) { return __builtin_popcountll(x); }
constexpr u64 EVEN = 0x5555555555555555ULL;

// ------------------------------------------------------------ host algebra
// Phase exponent p of G*K = i^p (G xor K); the same formulas as the device
// (crates/pauli/src/algebra.rs:206-213, crates/majorana/src/algebra.rs:180-193).
int host_product_exp(int alg, int W, const u64* g, const u64* k) {
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
bool host_anticommutes(int alg, int W, const u64* g, const u64* k) {
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
int host_support(int W, const u64* k) {
  int n = 0;
  for (int i = 0; i < W; ++i) n += hpopc((k[i] | (k[i] >> 1)) & EVEN);
  return n;
}
u32 host_weight(int alg, int W, const u64* k, u32 n_units) {
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
  // apply_rows (tableau.rs:109-143) with phases as exponents of i.
  int apply(const std::vector<u64>& img, const std::vector<int>& sgn, const u64* mono, u64* out) const {
    std::vector<u64> src(W, 0), e(W, 0), g(W);
    for (int i = 0; i < W; ++i) out[i] = 0;
    int se = 0, ie = 0;
    for (int wi = 0; wi < W; ++wi) {
      u64 bits = mono[wi];
      while (bits) {
        int b = __builtin_ctzll(bits);
        bits &= bits - 1;
        size_t p = (size_t)wi * 64 + b;
        if (p >= rows) continue;
        std::fill(e.begin(), e.end(), 0);
        e[wi] = 1ULL << b;
        se += host_product_exp(alg, W, e.data(), src.data());
        src[wi] ^= e[wi];
        for (int i = 0; i < W; ++i) g[i] = img[p * W + i];
        ie += host_product_exp(alg, W, g.data(), out) + (sgn[p] < 0 ? 2 : 0);
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
    std::vector<u64> e(W), img(W);
    for (size_t p = 0; p < lim; ++p) {
      std::fill(e.begin(), e.end(), 0);
      e[p / 64] = 1ULL << (p % 64);
      if (!host_anticommutes(alg, W, gen, e.data())) continue;
      int pe = host_product_exp(alg, W, gen, e.data());
      for (int i = 0; i < W; ++i) img[i] = gen[i] ^ e[i];
      // sign = sin * (-Im i^p); the rotation is Clifford so |sin| rounds to 1.
      double nim = pe == 1 ? -1.0 : (pe == 3 ? 1.0 : 0.0);
      double sign = sn * nim;
      int s = sign < 0 ? -1 : 1;
      for (int i = 0; i < W; ++i) t.rd_img[p * W + i] = t.gen_img[p * W + i] = img[i];
      t.rd_sign[p] = s;
      t.gen_sign[p] = -s;
    }
    t.refresh_identity();
    return t;
  }
  // changes_weight of for_rotation(gen) without building the tableau: a
  // single-bit row keeps its image unless it anticommutes with gen, and then
  // its image is gen ^ e_p.
  static bool rotation_changes_weight(int alg, int W, u32 n_units, const u64* gen) {
    const size_t lim = std::min((size_t)2 * n_units, (size_t)64 * W);
    u64 e[64] = {0}, img[64];
    for (size_t p = 0; p < lim; ++p) {
      e[p / 64] = 1ULL << (p % 64);
      const bool anti = host_anticommutes(alg, W, gen, e);
      e[p / 64] = 0;
      if (!anti) continue;
      for (int i = 0; i < W; ++i) img[i] = gen[i];
      img[p / 64] ^= 1ULL << (p % 64);
      if (host_support(W, img) != 1) return true;
    }
    return false;
  }
  bool changes_weight() const {
    for (size_t p = 0; p < rows; ++p) {
      std::vector<u64> u(W, 0);
      if (p < (size_t)64 * W) u[p / 64] = 1ULL << (p % 64);
      if (host_support(W, &rd_img[p * W]) != host_support(W, u.data())) return true;
    }
    return false;
  }
};

// --------------------------------------------------------------- plugins
struct Plugin {
  bool noise = true;
  void* lib = nullptr;
  void* ctx = nullptr;
  u32 depends = 0;
  void* fn = nullptr;
  void* batch_fn = nullptr;
  void (*destroy)(void*) = nullptr;
  ~Plugin() {
    if (destroy) destroy(ctx);
    if (lib) dlclose(lib);
  }
};
typedef double (*NoiseFactorFn)(void*, u32, const u64*, size_t, u32, u32, u32, u32);
typedef int32_t (*KeepFn)(void*, u32, const u64*, size_t, u32, u32, double, u32, u32);

void set_err(char* err, size_t n, const std::string& m) {
  if (err && n) snprintf(err, n, "%s", m.c_str());
}

// The reference loader's checks and messages (native_noise.rs:217-288,
// native_truncator.rs:205-276, depends_from_bits :350-357).
int load_plugin(bool noise, const char* path, const char* config, pq_plugin** out, char* err, size_t n) {
  const std::string kind = noise ? "noise" : "truncator";
  const std::string pre = noise ? "propaq_noise_" : "propaq_truncator_";
  void* lib = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!lib) {
    set_err(err, n, "failed to load " + kind + " plugin '" + path + "': " + dlerror());
    return PQ_ERR_PLUGIN_LOAD;
  }
  auto sym = [&](const char* s) { return dlsym(lib, (pre + s).c_str()); };
  auto fail = [&](const std::string& m) {
    dlclose(lib);
    set_err(err, n, m);
    return PQ_ERR_PLUGIN;
  };
  auto abi = (u32(*)(void))sym("abi_version");
  if (!abi) return fail(kind + " plugin '" + path + "' does not export " + pre + "abi_version");
  u32 v = abi();
  if (v != 1)
    return fail(kind + " plugin '" + path + "' targets ABI version " + std::to_string(v) + ", expected 1");
  u32 dep = 0;
  if (auto d = (u32(*)(void))sym("depends")) {
    dep = d();
    if (dep & ~3u) {
      char b[32];
      snprintf(b, sizeof b, "%#x", dep);
      return fail(kind + " plugin '" + path + "' declares unknown dependency bits " + b +
                  " (this build understands 0x3); it was likely built against a newer propaq");
    }
  }
  void* fn = sym(noise ? "factor" : "keep");
  if (!fn) return fail(kind + " plugin '" + path + "' does not export " + pre + (noise ? "factor" : "keep"));
  void* bfn = sym(noise ? "factor_batch" : "keep_batch");
  auto create = (void* (*)(const char*))sym("create");
  auto destroy = (void (*)(void*))sym("destroy");
  if ((create != nullptr) != (destroy != nullptr))
    return fail(kind + " plugin '" + path + "' must export both " + pre + "create and " + pre +
                "destroy, or neither");
  auto* p = new Plugin();
  p->noise = noise;
  p->lib = lib;
  p->depends = dep;
  p->fn = fn;
  p->batch_fn = bfn;
  p->destroy = destroy;
  p->ctx = create ? create(config) : nullptr;
  *out = reinterpret_cast<pq_plugin*>(p);
  return PQ_OK;
}

u64 next_pow2(u64 x) {
  u64 p = 1;
  while (p < x) p <<= 1;
  return p;
}

}  // namespace

// ---------------------------------------------------------------- engine
struct pq_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_begin = nullptr, ev_end = nullptr, ev_l0 = nullptr, ev_l1 = nullptr;
  std::string err;
  pq::SweepState* st = nullptr;    // device
  pq::SweepState* h_st = nullptr;  // pinned mirror
  u64* keys[2] = {nullptr, nullptr};
  double* coeffs[2] = {nullptr, nullptr};
  u64* table = nullptr;
  u64 tcap = 0;
  u64* status = nullptr;
  u64 cap = 0;
  int W = 0;
  int cur = 0;
  u32 epoch_base = 1;
  // per-op device arrays
  size_t ops_cap = 0;
  pq::OpDesc* d_ops = nullptr;
  u32* tickets = nullptr;
  u64* hist = nullptr;
  u64* anti = nullptr;
  u64* stamps = nullptr;
  void* d_gates = nullptr;
  size_t gates_bytes = 0;
  double* d_tables = nullptr;
  size_t d_tables_cap = 0;
  pq::ExpectPartial* partials = nullptr;
  int expect_grid = 0;
  u32* d_err = nullptr;  // error word of the stand-alone kernels
  std::vector<u64> out_keys;
  std::vector<double> out_coeffs;
  u64 launches = 0;

  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
  int cuda_fail(cudaError_t e, const char* what) {
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? PQ_ERR_OOM : PQ_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
  }
  void free_rows() {
    for (int i = 0; i < 2; ++i) {
      if (keys[i]) cudaFree(keys[i]);
      if (coeffs[i]) cudaFree(coeffs[i]);
      keys[i] = nullptr;
      coeffs[i] = nullptr;
    }
    if (table) cudaFree(table);
    if (status) cudaFree(status);
    table = nullptr;
    status = nullptr;
    cap = tcap = 0;
  }
  void free_ops() {
    for (void* p : {(void*)d_ops, (void*)tickets, (void*)hist, (void*)anti, (void*)stamps})
      if (p) cudaFree(p);
    d_ops = nullptr;
    tickets = nullptr;
    hist = anti = stamps = nullptr;
    ops_cap = 0;
  }
  ~pq_engine() {
    if (stream) cudaStreamSynchronize(stream);
    free_rows();
    free_ops();
    for (void* p : {(void*)st, (void*)d_gates, (void*)d_tables, (void*)partials, (void*)d_err})
      if (p) cudaFree(p);
    if (h_st) cudaFreeHost(h_st);
    for (auto ev : {ev_begin, ev_end, ev_l0, ev_l1})
      if (ev) cudaEventDestroy(ev);
    if (stream) cudaStreamDestroy(stream);
  }
  // (Re)allocates rows for `new_cap`, keeping the first n live rows of buffer
  // `from` in buffer 0, then clears and rebuilds the table.  Synchronous.
  int resize(u64 new_cap, u64 n, int from, int Wn) {
    cudaError_t e;
    u64* nk[2] = {nullptr, nullptr};
    double* nc[2] = {nullptr, nullptr};
    const u64 ntcap = 2 * new_cap;
    u64* nt = nullptr;
    u64* ns = nullptr;
    const u64 n_status = new_cap / TILE_ROWS + 2;
    auto cleanup = [&]() {
      for (int i = 0; i < 2; ++i) {
        if (nk[i]) cudaFree(nk[i]);
        if (nc[i]) cudaFree(nc[i]);
      }
      if (nt) cudaFree(nt);
      if (ns) cudaFree(ns);
    };
    for (int i = 0; i < 2; ++i) {
      if ((e = cudaMalloc(&nk[i], new_cap * Wn * 8)) != cudaSuccess ||
          (e = cudaMalloc(&nc[i], new_cap * 8)) != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "allocating term rows");
      }
    }
    if ((e = cudaMalloc(&nt, ntcap * 8)) != cudaSuccess || (e = cudaMalloc(&ns, n_status * 8)) != cudaSuccess) {
      cleanup();
      return cuda_fail(e, "allocating the hash table");
    }
    if (n && keys[from]) {
      cudaMemcpyAsync(nk[0], keys[from], n * Wn * 8, cudaMemcpyDeviceToDevice, stream);
      cudaMemcpyAsync(nc[0], coeffs[from], n * 8, cudaMemcpyDeviceToDevice, stream);
    }
    cudaMemsetAsync(ns, 0, n_status * 8, stream);
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) {
      cleanup();
      return cuda_fail(e, "copying rows");
    }
    free_rows();
    keys[0] = nk[0];
    keys[1] = nk[1];
    coeffs[0] = nc[0];
    coeffs[1] = nc[1];
    table = nt;
    status = ns;
    cap = new_cap;
    tcap = ntcap;
    cur = 0;
    W = Wn;
    return rebuild_table(n);
  }
  int rebuild_table(u64 n) {
    cudaMemsetAsync(table, 0xff, tcap * 8, stream);
    cudaError_t e;
    switch (W) {
      case 1: e = pq::launch_rebuild<1>(keys[cur], n, table, tcap - 1, d_err, stream); break;
      case 2: e = pq::launch_rebuild<2>(keys[cur], n, table, tcap - 1, d_err, stream); break;
      case 4: e = pq::launch_rebuild<4>(keys[cur], n, table, tcap - 1, d_err, stream); break;
      default: e = pq::launch_rebuild<8>(keys[cur], n, table, tcap - 1, d_err, stream); break;
    }
    if (n) ++launches;
    if (e != cudaSuccess) return cuda_fail(e, "rebuild launch");
    return PQ_OK;
  }
  int ensure_ops(size_t n_ops) {
    if (ops_cap >= n_ops) return PQ_OK;
    free_ops();
    cudaError_t e;
    if ((e = cudaMalloc(&d_ops, n_ops * sizeof(pq::OpDesc))) != cudaSuccess ||
        (e = cudaMalloc(&tickets, n_ops * 4)) != cudaSuccess || (e = cudaMalloc(&hist, n_ops * 8)) != cudaSuccess ||
        (e = cudaMalloc(&anti, n_ops * 8)) != cudaSuccess || (e = cudaMalloc(&stamps, n_ops * 8)) != cudaSuccess)
      return cuda_fail(e, "allocating op arrays");
    ops_cap = n_ops;
    return PQ_OK;
  }
};

namespace {

template <int W>
pq::GenInfo<W> make_gen(int alg, const u64* g, int sign) {
  pq::GenInfo<W> gi;
  int aux = 0;
  for (int i = 0; i < W; ++i) {
    gi.gen[i] = g[i];
    gi.fold[i] = alg == 0 ? (((g[i] & EVEN) << 1) | ((g[i] >> 1) & EVEN)) : g[i];
    aux += alg == 0 ? hpopc(g[i] & (g[i] >> 1) & EVEN) : hpopc(g[i]);
  }
  gi.aux = aux;
  gi.sign = sign < 0 ? -1.0 : 1.0;
  gi.carry = 0;
  int above = 0;
  for (int i = W - 1; i >= 0; --i) {
    u64 s = g[i] >> 1;
    for (int sh = 1; sh < 64; sh <<= 1) s ^= s >> sh;
    gi.sfx[i] = s;
    if (above) gi.carry |= 1u << i;
    above ^= hpopc(g[i]) & 1;
  }
  return gi;
}

template <int W, int ALG>
int run_impl(pq_engine* E, const pq_run_config* cfg, const u64* obs_words, const double* obs_coeffs, size_t n_obs,
             const u64* gate_words, const double* angles, size_t n_gates, const u32* layer_off, size_t n_layers,
             const u64* diag, size_t nd, u64* n_terms_out, pq_result* res) {
  const u32 n_units = cfg->n_units;
  const bool has_w = cfg->max_weight >= 0;
  const u32 wcut = has_w ? (u32)std::min<int64_t>(cfg->max_weight, 0xfffffffe) : pq::NO_WEIGHT_CUT;
  const bool has_c = cfg->has_min_coeff != 0;
  const double ccut = cfg->min_coeff;
  const bool has_floor = cfg->min_terms >= 0;
  const u64 floor_terms = has_floor ? (u64)cfg->min_terms : 0;
  cudaError_t e;

  // Noise resolution (noise_resolver.rs:78-131): one factor table per layer
  // or one for the run.
  const Plugin* np = reinterpret_cast<const Plugin*>(cfg->noise_plugin);
  size_t tlen = cfg->noise_table_len ? cfg->noise_table_len : (size_t)n_units + 1;
  std::vector<double> tables;
  bool layered = false;
  const bool have_noise = cfg->noise_kind != PQ_NOISE_NONE;
  if (cfg->noise_kind == PQ_NOISE_TABLE) {
    if (!cfg->noise_tables || !cfg->noise_table_len) return E->fail(PQ_ERR_INVALID, "noise table missing");
    tables.assign(cfg->noise_tables, cfg->noise_tables + tlen);
  } else if (cfg->noise_kind == PQ_NOISE_LAYERED) {
    if (!cfg->noise_tables || !cfg->noise_table_len) return E->fail(PQ_ERR_INVALID, "noise tables missing");
    tables.assign(cfg->noise_tables, cfg->noise_tables + tlen * n_layers);
    layered = true;
  } else if (cfg->noise_kind == PQ_NOISE_PLUGIN) {
    if (!np) return E->fail(PQ_ERR_INVALID, "noise plugin missing");
    if (np->depends & 1)
      return E->fail(PQ_ERR_UNSUPPORTED, "key-reading noise plugins are not run by the CUDA engine yet");
    tlen = (size_t)n_units + 1;
    auto f = (NoiseFactorFn)np->fn;
    auto tab = [&](u32 layer, u32 total) {
      for (u32 w = 0; w < n_units + 1; ++w) tables.push_back(f(np->ctx, ALG, nullptr, 0, n_units, w, layer, total));
    };
    if (np->depends & 2) {
      layered = true;
      for (size_t l = 0; l < n_layers; ++l) tab((u32)l, (u32)n_layers);
    } else {
      tab(0, 0);
    }
  } else if (cfg->noise_kind != PQ_NOISE_NONE) {
    return E->fail(PQ_ERR_INVALID, "unknown noise kind");
  }
  if (cfg->truncator)
    return E->fail(PQ_ERR_UNSUPPORTED, "native truncator plugins are not run by the CUDA engine yet");

  // Observable admission with duplicate folding (engine.rs:104-111).
  std::vector<u64> hk;
  std::vector<double> hc;
  {
    struct H {
      size_t operator()(const std::vector<u64>& v) const { return (size_t)pq::key_hash<W>(v.data()); }
    };
    std::unordered_map<std::vector<u64>, size_t, H> pos;
    std::vector<u64> k(W);
    for (size_t i = 0; i < n_obs; ++i) {
      std::memcpy(k.data(), obs_words + i * W, 8 * W);
      const double c = obs_coeffs[i];
      if (has_w && host_weight(ALG, W, k.data(), n_units) > wcut) continue;
      if (has_c && !(std::fabs(c) >= ccut)) continue;
      auto it = pos.find(k);
      if (it != pos.end()) {
        hc[it->second] += c;
      } else {
        pos.emplace(k, hc.size());
        hk.insert(hk.end(), k.begin(), k.end());
        hc.push_back(c);
      }
    }
  }
  const u64 n0 = hc.size();

  // Device set-up: rows, table, op arrays, noise tables.
  const u64 want_cap = next_pow2(std::max<u64>(4 * n0, 1ULL << 16));
  if (E->W != W || E->cap < want_cap) {
    if (int rc = E->resize(std::max(want_cap, E->cap), 0, E->cur, W)) return rc;
  }
  E->cur = 0;
  if (n0) {
    cudaMemcpyAsync(E->keys[0], hk.data(), n0 * W * 8, cudaMemcpyHostToDevice, E->stream);
    cudaMemcpyAsync(E->coeffs[0], hc.data(), n0 * 8, cudaMemcpyHostToDevice, E->stream);
  }
  if (int rc = E->rebuild_table(n0)) return rc;
  const size_t n_ops_max = n_gates + n_layers + 1;
  if (int rc = E->ensure_ops(n_ops_max)) return rc;
  const size_t gbytes = std::max<size_t>(n_gates, 1) * sizeof(pq::GateDesc<W>);
  if (E->gates_bytes < gbytes) {
    if (E->d_gates) cudaFree(E->d_gates);
    E->d_gates = nullptr;
    if ((e = cudaMalloc(&E->d_gates, gbytes)) != cudaSuccess) return E->cuda_fail(e, "gate descriptors");
    E->gates_bytes = gbytes;
  }
  if (!tables.empty() && E->d_tables_cap < tables.size()) {
    if (E->d_tables) cudaFree(E->d_tables);
    E->d_tables = nullptr;
    if ((e = cudaMalloc(&E->d_tables, tables.size() * 8)) != cudaSuccess) return E->cuda_fail(e, "noise tables");
    E->d_tables_cap = tables.size();
  }
  if (!tables.empty())
    cudaMemcpyAsync(E->d_tables, tables.data(), tables.size() * 8, cudaMemcpyHostToDevice, E->stream);
  cudaMemsetAsync(E->anti, 0, n_ops_max * 8, E->stream);
  if (E->epoch_base > (1u << 29)) {  // keep status tags unique: restart the epochs on a cleared array
    E->epoch_base = 1;
    cudaMemsetAsync(E->status, 0, (E->cap / TILE_ROWS + 2) * 8, E->stream);
  }

  std::vector<pq::OpDesc> ops;
  std::vector<pq::GateDesc<W>> gdesc;
  ops.reserve(n_ops_max);
  gdesc.reserve(n_gates);
  std::vector<long> gate_op(n_gates, -1);  // latest op at or before each gate
  u64 n_live = n0, peak = n0;
  size_t done = 0;  // ops executed so far
  size_t gdone = 0; // gate descriptors uploaded so far
  const int grid = pq::sweep_grid<W, ALG>((int)cfg->blocks_per_sm);
  double sweep_ms = 0;
  u64 sweep_launches = 0;
  bool began = false;

  // Runs ops [done, ops.size()) on the device; on a capacity halt grows the
  // rows and relaunches from the halted op.
  auto flush = [&]() -> int {
    if (ops.size() > done) {
      cudaMemcpyAsync(E->d_ops + done, ops.data() + done, (ops.size() - done) * sizeof(pq::OpDesc),
                      cudaMemcpyHostToDevice, E->stream);
    }
    if (gdesc.size() > gdone) {
      cudaMemcpyAsync(reinterpret_cast<pq::GateDesc<W>*>(E->d_gates) + gdone, gdesc.data() + gdone,
                      (gdesc.size() - gdone) * sizeof(pq::GateDesc<W>), cudaMemcpyHostToDevice, E->stream);
      gdone = gdesc.size();
    }
    while (done < ops.size()) {
      pq::SweepState s{};
      s.n[done & 1] = n_live;
      s.peak = peak;
      s.halt = pq::NOT_HALTED;
      s.bar_gen = 0;
      *E->h_st = s;
      cudaMemcpyAsync(E->st, E->h_st, sizeof s, cudaMemcpyHostToDevice, E->stream);
      cudaMemsetAsync(E->tickets + done, 0, (ops.size() - done) * 4, E->stream);
      pq::SweepArgs a{};
      a.ops = E->d_ops;
      a.gates = E->d_gates;
      a.tables = E->d_tables;
      a.table_len = (u32)tlen;
      a.n_units = n_units;
      a.op_begin = (u32)done;
      a.op_end = (u32)ops.size();
      a.cur0 = (u32)E->cur;
      a.epoch_base = E->epoch_base;
      a.max_weight = wcut;
      a.has_min_coeff = has_c;
      a.min_coeff = ccut;
      a.min_terms = floor_terms;
      for (int i = 0; i < 2; ++i) {
        a.keys[i] = E->keys[i];
        a.coeffs[i] = E->coeffs[i];
      }
      a.table = E->table;
      a.table_mask = E->tcap - 1;
      a.cap = E->cap;
      a.status = E->status;
      a.tickets = E->tickets;
      a.hist = E->hist;
      a.anti = E->anti;
      a.stamps = E->stamps;
      a.st = E->st;
      if (!began) {  // device time starts at the first sweep
        cudaEventRecord(E->ev_begin, E->stream);
        began = true;
      }
      cudaEventRecord(E->ev_l0, E->stream);
      if ((e = pq::launch_sweep<W, ALG>(a, grid, E->stream)) != cudaSuccess) return E->cuda_fail(e, "sweep launch");
      cudaEventRecord(E->ev_l1, E->stream);
      ++E->launches;
      ++sweep_launches;
      E->epoch_base += (u32)ops.size() + 1;
      cudaMemcpyAsync(E->h_st, E->st, sizeof s, cudaMemcpyDeviceToHost, E->stream);
      if ((e = cudaStreamSynchronize(E->stream)) != cudaSuccess) return E->cuda_fail(e, "sweep");
      float ms = 0;
      cudaEventElapsedTime(&ms, E->ev_l0, E->ev_l1);
      sweep_ms += ms;
      const pq::SweepState h = *E->h_st;
      if (h.error & pq::ERR_BARRIER_TIMEOUT)
        return E->fail(PQ_ERR_DEVICE_TIMEOUT, "a grid barrier wait expired on the device");
      if (h.error & pq::ERR_LOOKBACK_TIMEOUT)
        return E->fail(PQ_ERR_DEVICE_TIMEOUT, "a tile's look-back wait expired on the device");
      if (h.error) return E->fail(PQ_ERR_CUDA, "device reported error bits " + std::to_string(h.error));
      E->cur = (int)h.cur;
      done = h.end_op;
      n_live = h.n[done & 1];
      peak = std::max(peak, h.peak);
      if (h.halt != pq::NOT_HALTED) {  // grow: the gate at `done` needs 2 N rows
        u64 ncap = next_pow2(std::max<u64>(4 * n_live, 2 * E->cap));
        if (ncap > MAX_ROWS) ncap = MAX_ROWS;
        if (2 * n_live > ncap)
          return E->fail(PQ_ERR_CEILING, "term index ceiling reached: " + std::to_string(2 * n_live) +
                                             " rows would exceed the engine's capacity");
        int rc = E->resize(ncap, n_live, E->cur, W);
        if (rc == PQ_ERR_OOM) rc = E->resize(next_pow2(2 * n_live), n_live, E->cur, W);
        if (rc) return rc;
      }
    }
    return PQ_OK;
  };

  Tableau frame(ALG, W, n_units);
  std::vector<u64> g(W), gc(W);
  long last_op = -1;
  for (size_t l = 0; l < n_layers; ++l) {
    if (have_noise) {
      pq::OpDesc od;
      od.kind = (has_w || has_c) ? pq::OP_NOISE_COMPACT : pq::OP_NOISE_SCALE;  // partitioned_termsum.rs:585-587
      od.idx = layered ? (u32)l : 0u;
      ops.push_back(od);
      last_op = (long)ops.size() - 1;
    }
    for (u32 gi = layer_off[l]; gi < layer_off[l + 1]; ++gi) {
      std::memcpy(g.data(), gate_words + (size_t)gi * W, 8 * W);
      const double ang = angles[gi];
      if (std::fabs(std::cos(ang)) < EPS_CLASSIFY) {  // Clifford: defer into the frame when allowed
        bool eff_w = has_w;
        const bool cw = Tableau::rotation_changes_weight(ALG, W, n_units, g.data());
        if (has_w && cw && has_floor) {  // the effective cutoff depends on the live count here
          if (int rc = flush()) return rc;
          if (n_live < floor_terms) eff_w = false;
        }
        if (!eff_w || !cw) {
          frame.compose(Tableau::for_rotation(ALG, W, n_units, g.data(), ang));
          gate_op[gi] = last_op;
          continue;
        }
      }
      const int sign = frame.conjugate_generator(g.data(), gc.data());
      pq::GateDesc<W> gd;
      gd.g = make_gen<W>(ALG, gc.data(), sign);
      gd.sn = std::sin(ang);
      gd.cs = std::cos(ang);
      pq::OpDesc od;
      od.kind = std::fabs(gd.sn) < EPS_CLASSIFY ? pq::OP_PHASE : pq::OP_GATE;
      od.idx = (u32)gdesc.size();
      gdesc.push_back(gd);
      ops.push_back(od);
      last_op = (long)ops.size() - 1;
      gate_op[gi] = last_op;
    }
  }
  if (int rc = flush()) return rc;
  if (!began) cudaEventRecord(E->ev_begin, E->stream);
  const u64 n_fin = n_live;

  std::vector<u64> hist(ops.size()), anti(ops.size()), stamps(ops.size());
  if (!ops.empty()) {
    cudaMemcpyAsync(hist.data(), E->hist, ops.size() * 8, cudaMemcpyDeviceToHost, E->stream);
    cudaMemcpyAsync(anti.data(), E->anti, ops.size() * 8, cudaMemcpyDeviceToHost, E->stream);
    cudaMemcpyAsync(stamps.data(), E->stamps, ops.size() * 8, cudaMemcpyDeviceToHost, E->stream);
  }

  // Expectation value and the below-cutoff count.
  res->expectation_value = 0;
  res->terms_below_cutoff = 0;
  u64* d_img = nullptr;
  int* d_sgn = nullptr;
  struct FrameFree {
    u64** a;
    int** b;
    ~FrameFree() {
      if (*a) cudaFree(*a);
      if (*b) cudaFree(*b);
    }
  } ff{&d_img, &d_sgn};
  if (!frame.identity) {
    if ((e = cudaMalloc(&d_img, frame.rd_img.size() * 8)) != cudaSuccess) return E->cuda_fail(e, "frame");
    if ((e = cudaMalloc(&d_sgn, frame.rd_sign.size() * sizeof(int))) != cudaSuccess) return E->cuda_fail(e, "frame");
    cudaMemcpyAsync(d_img, frame.rd_img.data(), frame.rd_img.size() * 8, cudaMemcpyHostToDevice, E->stream);
    cudaMemcpyAsync(d_sgn, frame.rd_sign.data(), frame.rd_sign.size() * sizeof(int), cudaMemcpyHostToDevice,
                    E->stream);
  }
  if (diag || has_c) {
    pq::ExpectArgs xa{};
    if (diag) {
      for (u32 u = 0; u < n_units; ++u) {
        const u64 bit = (u / 64 < nd) ? (diag[u / 64] >> (u % 64)) & 1 : 0;
        if (!bit) continue;
        const u32 pos = ALG == 0 ? 2 * u + 1 : 2 * u;
        if (pos / 64 < (u32)W) xa.state[pos / 64] |= 1ULL << (pos % 64);
      }
    }
    xa.n_units = n_units;
    xa.has_min_coeff = has_c;
    xa.min_coeff = ccut;
    xa.frame_images = d_img;
    xa.frame_signs = d_sgn;
    xa.frame_rows = (u32)frame.rows;
    ++E->launches;
    if ((e = pq::launch_expect<W, ALG>(xa, E->keys[E->cur], E->coeffs[E->cur], n_fin, E->partials, E->expect_grid,
                                       E->stream)) != cudaSuccess)
      return E->cuda_fail(e, "expectation launch");
    cudaEventRecord(E->ev_end, E->stream);
    std::vector<pq::ExpectPartial> parts(E->expect_grid);
    cudaMemcpyAsync(parts.data(), E->partials, parts.size() * sizeof(pq::ExpectPartial), cudaMemcpyDeviceToHost,
                    E->stream);
    if ((e = cudaStreamSynchronize(E->stream)) != cudaSuccess) return E->cuda_fail(e, "expectation");
    double hi = 0, lo = 0;
    auto dd = [&](double v) {
      const double s = hi + v, bb = s - hi;
      double er = (hi - (s - bb)) + (v - bb);
      er += lo;
      hi = s + er;
      lo = er - (hi - s);
    };
    u64 below = 0;
    for (auto& p : parts) {
      dd(p.hi);
      dd(p.lo);
      below += p.below;
    }
    if (diag) res->expectation_value = hi + lo;
    res->terms_below_cutoff = has_c ? below : 0;
  } else {
    cudaEventRecord(E->ev_end, E->stream);
    if ((e = cudaStreamSynchronize(E->stream)) != cudaSuccess) return E->cuda_fail(e, "sync");
  }

  if (n_terms_out)
    for (size_t gi = 0; gi < n_gates; ++gi) n_terms_out[gi] = gate_op[gi] >= 0 ? hist[gate_op[gi]] : n0;

  E->out_keys.clear();
  E->out_coeffs.clear();
  if (cfg->want_terms && n_fin) {
    E->out_keys.resize(n_fin * W);
    E->out_coeffs.resize(n_fin);
    if (frame.identity) {
      cudaMemcpyAsync(E->out_keys.data(), E->keys[E->cur], n_fin * W * 8, cudaMemcpyDeviceToHost, E->stream);
      cudaMemcpyAsync(E->out_coeffs.data(), E->coeffs[E->cur], n_fin * 8, cudaMemcpyDeviceToHost, E->stream);
    } else {
      // The alternate buffer is free after the sweep: conjugate into it.
      const int alt = E->cur ^ 1;
      ++E->launches;
      pq::launch_conjugate<W>(E->keys[E->cur], E->coeffs[E->cur], n_fin, d_img, d_sgn, (u32)frame.rows, ALG,
                              E->keys[alt], E->coeffs[alt], E->stream);
      cudaMemcpyAsync(E->out_keys.data(), E->keys[alt], n_fin * W * 8, cudaMemcpyDeviceToHost, E->stream);
      cudaMemcpyAsync(E->out_coeffs.data(), E->coeffs[alt], n_fin * 8, cudaMemcpyDeviceToHost, E->stream);
    }
    if ((e = cudaStreamSynchronize(E->stream)) != cudaSuccess) return E->cuda_fail(e, "terms copy");
  }

  // Per-kind totals (inputs of the algorithmic-bytes roofline) and the
  // device-clock split of the sweep time by op kind.
  for (size_t i = 0; i < ops.size(); ++i) {
    const u64 n_in = i ? hist[i - 1] : n0;
    const double op_ms = i ? (double)(stamps[i] - stamps[i - 1]) * 1e-6 : 0.0;
    switch (ops[i].kind) {
      case pq::OP_GATE:
        ++res->gate_ops;
        res->gate_ms += op_ms;
        res->sum_rows_gate += n_in;
        res->sum_anti += anti[i];
        res->sum_children += hist[i] - n_in;
        break;
      case pq::OP_PHASE:
        ++res->phase_ops;
        res->phase_ms += op_ms;
        res->sum_rows_phase += n_in;
        break;
      default:
        ++res->noise_ops;
        res->noise_ms += op_ms;
        res->sum_rows_noise += n_in;
        res->sum_kept += ops[i].kind == pq::OP_NOISE_COMPACT ? hist[i] : 0;
    }
  }
  float ms = 0;
  cudaEventElapsedTime(&ms, E->ev_begin, E->ev_end);
  res->device_ms = ms;
  res->sweep_ms = sweep_ms;
  res->sweep_launches = sweep_launches;
  res->n_final = n_fin;
  res->peak_terms = peak;
  res->sparse_key_bytes = n_fin * W * 8 + E->tcap * 8;
  res->n_layers_run = n_layers;
  res->n_gates_run = n_gates;
  return PQ_OK;
}

template <int W>
int run_alg(pq_engine* E, const pq_run_config* c, const u64* ow, const double* oc, size_t no, const u64* gw,
            const double* ga, size_t ng, const u32* lo, size_t nl, const u64* d, size_t nd, u64* nt,
            pq_result* r) {
  if (c->basis_kind == PQ_BASIS_PAULI) return run_impl<W, 0>(E, c, ow, oc, no, gw, ga, ng, lo, nl, d, nd, nt, r);
  return run_impl<W, 1>(E, c, ow, oc, no, gw, ga, ng, lo, nl, d, nd, nt, r);
}

}  // namespace

extern "C" {

uint32_t pq_words_for_units(uint32_t n) {
  if (n > MAX_UNITS) return 0;
  uint32_t w = 1;
  while ((uint64_t)32 * w < n) w <<= 1;
  return w;
}

int pq_engine_create(pq_engine** out, int device) {
  *out = nullptr;
  auto E = std::make_unique<pq_engine>();
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count <= device || device < 0) {
    cudaGetLastError();
    return PQ_ERR_CUDA;
  }
  if ((e = cudaSetDevice(device)) != cudaSuccess) return PQ_ERR_CUDA;
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
  if (!coop) return PQ_ERR_CUDA;
  E->device = device;
  if (cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking) != cudaSuccess) return PQ_ERR_CUDA;
  if (cudaMalloc(&E->st, sizeof(pq::SweepState)) != cudaSuccess) return PQ_ERR_OOM;
  if (cudaMallocHost(&E->h_st, sizeof(pq::SweepState)) != cudaSuccess) return PQ_ERR_OOM;
  if (cudaMalloc(&E->d_err, sizeof(u32)) != cudaSuccess) return PQ_ERR_OOM;
  cudaMemset(E->d_err, 0, sizeof(u32));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  E->expect_grid = 4 * sms;
  if (cudaMalloc(&E->partials, sizeof(pq::ExpectPartial) * E->expect_grid) != cudaSuccess) return PQ_ERR_OOM;
  for (cudaEvent_t* ev : {&E->ev_begin, &E->ev_end, &E->ev_l0, &E->ev_l1}) cudaEventCreate(ev);
  *out = E.release();
  return PQ_OK;
}

void pq_engine_destroy(pq_engine* E) { delete E; }
const char* pq_engine_last_error(const pq_engine* E) { return E ? E->err.c_str() : "null engine"; }

int pq_run(pq_engine* E, const pq_run_config* cfg, const uint64_t* ow, const double* oc, size_t no,
           const uint64_t* gw, const double* ga, size_t ng, const uint32_t* lo, size_t nl, const uint64_t* d,
           size_t nd, uint64_t* nt, pq_result* r) {
  if (!E || !cfg || !r) return PQ_ERR_INVALID;
  std::memset(r, 0, sizeof(*r));
  E->err.clear();
  if (cfg->basis_kind > 1) return E->fail(PQ_ERR_INVALID, "basis_kind must be 0 (Pauli) or 1 (Majorana)");
  const uint32_t W = pq_words_for_units(cfg->n_units);
  if (!W)
    return E->fail(PQ_ERR_INVALID, "propaq: " + std::to_string(cfg->n_units) +
                                       " units exceeds the engine's maximum of 2048");
  if (nl && (!lo || lo[0] != 0 || lo[nl] != ng)) return E->fail(PQ_ERR_INVALID, "layer offsets do not cover the gates");
  for (size_t l = 0; l < nl; ++l)
    if (lo[l + 1] < lo[l]) return E->fail(PQ_ERR_INVALID, "layer offsets must be non-decreasing");
  if (cudaSetDevice(E->device) != cudaSuccess) return E->fail(PQ_ERR_CUDA, "cudaSetDevice failed");
  const u64 l0 = E->launches;
  // uint64_t and the kernels' unsigned long long are both 64-bit words.
  auto K = [](const uint64_t* p) { return reinterpret_cast<const u64*>(p); };
  auto Kw = reinterpret_cast<u64*>(nt);
  int rc;
  switch (W) {
    case 1: rc = run_alg<1>(E, cfg, K(ow), oc, no, K(gw), ga, ng, lo, nl, K(d), nd, Kw, r); break;
    case 2: rc = run_alg<2>(E, cfg, K(ow), oc, no, K(gw), ga, ng, lo, nl, K(d), nd, Kw, r); break;
    case 4: rc = run_alg<4>(E, cfg, K(ow), oc, no, K(gw), ga, ng, lo, nl, K(d), nd, Kw, r); break;
    case 8: rc = run_alg<8>(E, cfg, K(ow), oc, no, K(gw), ga, ng, lo, nl, K(d), nd, Kw, r); break;
    default:
      rc = E->fail(PQ_ERR_UNSUPPORTED, "registers wider than 256 units (" + std::to_string(W) +
                                           " words) are not compiled into this build");
  }
  r->gpu_launches = E->launches - l0;
  return rc;
}

size_t pq_result_terms(pq_engine* E, uint64_t* keys, double* coeffs, size_t cap) {
  const size_t n = E->out_coeffs.size();
  const size_t m = std::min(n, cap);
  if (m && E->W) {
    std::memcpy(keys, E->out_keys.data(), m * E->W * 8);
    std::memcpy(coeffs, E->out_coeffs.data(), m * 8);
  }
  return n;
}

int pq_plugin_load_noise(const char* path, const char* cfg, pq_plugin** out, char* err, size_t n) {
  return load_plugin(true, path, cfg, out, err, n);
}
int pq_plugin_load_truncator(const char* path, const char* cfg, pq_plugin** out, char* err, size_t n) {
  return load_plugin(false, path, cfg, out, err, n);
}
void pq_plugin_free(pq_plugin* p) { delete reinterpret_cast<Plugin*>(p); }
uint32_t pq_plugin_depends(const pq_plugin* p) { return reinterpret_cast<const Plugin*>(p)->depends; }
double pq_plugin_noise_factor(const pq_plugin* pp, uint32_t kind, const uint64_t* words, size_t nw, uint32_t n_units,
                              uint32_t weight, uint32_t layer, uint32_t n_layers) {
  auto* p = reinterpret_cast<const Plugin*>(pp);
  bool key = p->depends & 1;
  return ((NoiseFactorFn)p->fn)(p->ctx, kind, key ? reinterpret_cast<const u64*>(words) : nullptr, key ? nw : 0, n_units, weight, layer, n_layers);
}
int pq_plugin_truncator_keep(const pq_plugin* pp, uint32_t kind, const uint64_t* words, size_t nw, uint32_t n_units,
                             uint32_t weight, double mag, uint32_t layer, uint32_t n_layers) {
  auto* p = reinterpret_cast<const Plugin*>(pp);
  bool key = p->depends & 1;
  return ((KeepFn)p->fn)(p->ctx, kind, key ? reinterpret_cast<const u64*>(words) : nullptr, key ? nw : 0, n_units, weight, mag, layer, n_layers) !=
         0;
}

}  // extern "C"
