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
// The device side is one cooperative persistent launch per propagation (or
// per batch of propagations) that runs the whole op sequence with grid
// barriers between ops.  A gate that would need more rows than the buffers
// hold stops the launch and records where; the host grows the buffers,
// rebuilds the hash table and relaunches from that op.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../../include/propaq_cuda.h"
#include "pq_kernels.cuh"
#include "pq_sort.cuh"
#include "pq_tableau.h"

using pq::u32;
using pq::u64;
using pqh::EVEN;
using pqh::hpopc;
using pqh::host_anticommutes;
using pqh::host_product_exp;
using pqh::host_support;
using pqh::host_weight;
using pqh::Tableau;

namespace {

constexpr double EPS_CLASSIFY = 1e-9;  // termsum.rs:42, partitioned_termsum.rs:41
constexpr u32 MAX_UNITS = 2048;        // engine.rs:27
constexpr u64 MAX_ROWS = 1ULL << 31;   // row index ceiling of the table slots
constexpr int TILE_ROWS = 256;  // smallest tile a sweep uses (sizes the look-back status array)
// Observables of at least this many admitted terms fold their duplicate keys
// on the device (radix sort by key, then a sum over each run of equal keys);
// smaller ones on the host.
constexpr size_t DEVICE_FOLD_MIN = 1u << 15;

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
// The batch forms (native_noise.rs:142-188, native_truncator.rs:158-200): 0 = done.
typedef int32_t (*NoiseBatchFn)(void*, u32, const u64*, size_t, u32, const u32*, u32, u32, double*, size_t);
typedef int32_t (*KeepBatchFn)(void*, u32, const u64*, size_t, u32, const u32*, const double*, u32, u32, uint8_t*,
                               size_t);
constexpr size_t KERNEL_BATCH = 1024;  // term_kernel.rs:10

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

// Device allocations of an engine, counted against its budget
// (pq_engine_limits::max_device_bytes).  The entry points that act on an
// engine point t_budget at its budget for the duration of the call, so the
// helpers below need no engine argument; allocations made with no budget in
// force (or before a limit was set) are not counted.
struct MemBudget {
  size_t limit = 0, used = 0;  // limit 0 = none
  std::unordered_map<void*, size_t> sizes;
};
thread_local MemBudget* t_budget = nullptr;

struct BudgetScope {
  MemBudget* saved;
  explicit BudgetScope(MemBudget* b) : saved(t_budget) { t_budget = b; }
  ~BudgetScope() { t_budget = saved; }
};

template <class T>
cudaError_t dmalloc(T** p, size_t n) {
  *p = nullptr;
  MemBudget* b = t_budget;
  if (b && b->limit && b->used + n > b->limit) return cudaErrorMemoryAllocation;
  void* q = nullptr;
  const cudaError_t e = cudaMalloc(&q, n);
  if (e != cudaSuccess) return e;
  *p = static_cast<T*>(q);
  if (b) {
    b->used += n;
    b->sizes[q] = n;
  }
  return cudaSuccess;
}
inline void dfree(void* p) {
  if (!p) return;
  if (MemBudget* b = t_budget) {
    const auto it = b->sizes.find(p);
    if (it != b->sizes.end()) {
      b->used -= it->second;
      b->sizes.erase(it);
    }
  }
  cudaFree(p);
}

// ---------------------------------------------------------------- engine
namespace {

// Calls f(std::integral_constant<int, W>) for a compiled key width.
template <class F>
decltype(auto) with_words(int W, F&& f) {
  switch (W) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 8: return f(std::integral_constant<int, 8>{});
    case 16: return f(std::integral_constant<int, 16>{});
    case 32: return f(std::integral_constant<int, 32>{});
    default: return f(std::integral_constant<int, 64>{});
  }
}

// Device resources of one propagation.  Slot 0 serves pq_run; a batch uses
// slots 0..n-1.  Buffers grow on demand and are kept for the next run.
struct Slot {
  u64* keys[2] = {nullptr, nullptr};
  double* coeffs[2] = {nullptr, nullptr};
  u64* table = nullptr;
  u64 tcap = 0;
  u64 bmask = ~3ULL;  // ~(slots per table bucket - 1) of the run the slot holds
  u64* status = nullptr;
  u64 cap = 0;
  int W = 0;
  int cur = 0;
  u32 epoch_base = 1;
  size_t ops_cap = 0;
  pq::OpDesc* d_ops = nullptr;
  u32* tickets = nullptr;
  u64* hist = nullptr;
  u64* anti = nullptr;
  u64* stamps = nullptr;
  u64* logs = nullptr;  // per-op emit statistics of a logged run (LOG_WORDS per op)
  // class-op scratch (SweepArgs::cls_mask ...), sized to cap rows / tcap slots
  u64* cls_mask = nullptr;
  u32* cls_slot = nullptr;
  u32* cls_children = nullptr;
  u64* fam_table = nullptr;
  u64* fam_aux = nullptr;
  u64 cls_cap = 0, fam_cap = 0;
  bool fam_dirty = false;  // a launch failed part way: the family table may hold entries
  std::vector<pq_gate_record> gate_log;  // per-gate records of the last logged run
  void* d_gates = nullptr;
  size_t gates_bytes = 0;
  double* d_tables = nullptr;
  size_t d_tables_cap = 0;
  pq::ExpectPartial* partials = nullptr;
  u64* frame_img = nullptr;  // readout tableau of the last run, when not the identity
  int* frame_sgn = nullptr;
  size_t frame_cap = 0;
  unsigned char* host_state = nullptr;  // decisions made on the host for one op (see SweepArgs)
  double* host_factor = nullptr;
  unsigned char* host_keep = nullptr;
  size_t host_cap = 0;
  int out_words = 0;  // width of out_keys (the caller's width)
  std::vector<u64> out_keys;
  std::vector<double> out_coeffs;

  void free_rows() {
    for (int i = 0; i < 2; ++i) {
      if (keys[i]) dfree(keys[i]);
      if (coeffs[i]) dfree(coeffs[i]);
      keys[i] = nullptr;
      coeffs[i] = nullptr;
    }
    if (table) dfree(table);
    if (status) dfree(status);
    table = nullptr;
    status = nullptr;
    cap = tcap = 0;
  }
  void free_ops() {
    for (void* p : {(void*)d_ops, (void*)tickets, (void*)hist, (void*)anti, (void*)stamps, (void*)logs})
      if (p) dfree(p);
    d_ops = nullptr;
    tickets = nullptr;
    hist = anti = stamps = logs = nullptr;
    ops_cap = 0;
  }
  void free_class() {
    for (void* p : {(void*)cls_mask, (void*)cls_slot, (void*)cls_children, (void*)fam_table, (void*)fam_aux})
      if (p) dfree(p);
    cls_mask = nullptr;
    cls_slot = cls_children = nullptr;
    fam_table = fam_aux = nullptr;
    cls_cap = fam_cap = 0;
  }
  void free_all() {
    free_rows();
    free_ops();
    free_class();
    for (void* p : {(void*)d_gates, (void*)d_tables, (void*)partials, (void*)frame_img, (void*)frame_sgn,
                    (void*)host_state, (void*)host_factor, (void*)host_keep})
      if (p) dfree(p);
    host_state = nullptr;
    host_factor = nullptr;
    host_keep = nullptr;
    host_cap = 0;
    d_gates = nullptr;
    d_tables = nullptr;
    partials = nullptr;
    frame_img = nullptr;
    frame_sgn = nullptr;
    gates_bytes = d_tables_cap = frame_cap = 0;
  }
};

// Grows a device array (and its pinned host mirror, when `host` is given) to
// hold n elements.
template <class T>
cudaError_t grow_pair(T** dev, T** host, size_t* cap, size_t n) {
  if (*cap >= n) return cudaSuccess;
  if (*dev) dfree(*dev);
  if (host && *host) cudaFreeHost(*host);
  *dev = nullptr;
  if (host) *host = nullptr;
  *cap = 0;
  cudaError_t e = dmalloc(dev, n * sizeof(T));
  if (e == cudaSuccess && host) e = cudaMallocHost(host, n * sizeof(T));
  if (e == cudaSuccess) *cap = n;
  return e;
}

}  // namespace

// A grow-only device buffer the engine keeps between calls, carved into
// typed arrays by byte offset.  Released by the engine.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t n) {
    if (bytes >= n) return cudaSuccess;
    release();
    const cudaError_t e = dmalloc(&p, std::max<size_t>(n, 1));
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    bytes = n;
    return cudaSuccess;
  }
  void release() {
    if (p) dfree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T>
  T* at(size_t offset) const {
    return reinterpret_cast<T*>(static_cast<char*>(p) + offset);
  }
};
inline size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

struct pq_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_begin = nullptr, ev_end = nullptr, ev_l0 = nullptr, ev_l1 = nullptr;
  std::string err;
  std::vector<Slot> slots;
  pq::SweepState* d_states = nullptr;  // one per slot
  pq::SweepState* h_states = nullptr;  // pinned mirror
  size_t states_cap = 0;
  pq::SweepArgs* d_args = nullptr;  // per instance of a batched launch
  pq::SweepArgs* h_args = nullptr;
  size_t args_cap = 0;
  u32* d_block_inst = nullptr;  // instance of each block of a batched launch
  u32* h_block_inst = nullptr;
  size_t block_inst_cap = 0;
  int expect_grid = 0;
  u32* d_err = nullptr;   // error word of the stand-alone kernels
  u32* d_idle = nullptr;  // blocks left idle in a batched launch
  u64 launches = 0;
  // Gradient buffers (pq_run_adjoint), kept so that repeated gradients of
  // one problem allocate nothing: the record pool, the two adjoint vectors
  // and per-op arrays, the segment checkpoints, and the pool size the last
  // default-sized gradient needed to record every op.
  DevBuf g_pool, g_lam, g_ops;
  DevBuf sort_buf;  // radix-sort scratch and sorted rows (observable folding, sorted term output)
  std::vector<DevBuf> g_ck;
  size_t g_need = 0;
  // pq_engine_set_limits: the row ceiling, the device-memory budget the
  // engine's allocations count against, the device wait limits and the
  // failure tests' hold.
  pq_engine_limits lim{};
  MemBudget budget;

  // Largest row capacity a run may use: a power of two (the table is 2x the
  // rows and is indexed by mask), at most MAX_ROWS.
  u64 row_ceiling() const {
    const u64 m = lim.max_rows ? std::min<u64>(lim.max_rows, MAX_ROWS) : MAX_ROWS;
    u64 p = 1;
    while (2 * p <= m) p *= 2;
    return p;
  }
  void init_waits(pq::SweepState& st) const {
    st.barrier_limit = lim.barrier_spins ? lim.barrier_spins : pq::DEFAULT_BARRIER_POLLS;
    st.lookback_limit = lim.lookback_spins ? lim.lookback_spins : pq::DEFAULT_LOOKBACK_POLLS;
  }
  // The limits' share of a sweep launch's arguments.
  void limit_args(pq::SweepArgs& a) const {
    a.cap = std::min<u64>(a.cap, row_ceiling());
    a.hold_block = lim.hold_block;
    a.hold_us = std::min<u32>(lim.hold_us, 100000);
  }

  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
  int cuda_fail(cudaError_t e, const char* what) {
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? PQ_ERR_OOM : PQ_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
  }
  ~pq_engine() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto& s : slots) s.free_all();
    for (DevBuf* b : {&g_pool, &g_lam, &g_ops, &sort_buf}) b->release();
    for (DevBuf& b : g_ck) b.release();
    for (void* p : {(void*)d_states, (void*)d_args, (void*)d_block_inst, (void*)d_err, (void*)d_idle})
      if (p) dfree(p);
    for (void* p : {(void*)h_states, (void*)h_args, (void*)h_block_inst})
      if (p) cudaFreeHost(p);
    for (auto ev : {ev_begin, ev_end, ev_l0, ev_l1})
      if (ev) cudaEventDestroy(ev);
    if (stream) cudaStreamDestroy(stream);
  }
  int ensure_slots(size_t n) {
    if (slots.size() < n) slots.resize(n);
    if (cudaError_t e = grow_pair(&d_states, &h_states, &states_cap, n)) return cuda_fail(e, "sweep states");
    return PQ_OK;
  }
  int ensure_batch_arrays(size_t n_args, size_t n_blocks) {
    if (cudaError_t e = grow_pair(&d_args, &h_args, &args_cap, n_args)) return cuda_fail(e, "batch arguments");
    if (cudaError_t e = grow_pair(&d_block_inst, &h_block_inst, &block_inst_cap, n_blocks))
      return cuda_fail(e, "batch block map");
    return PQ_OK;
  }
  // (Re)allocates a slot's rows for `new_cap`, keeping the first n live rows
  // of buffer `from` in buffer 0, then clears and rebuilds the table.
  // Synchronous.
  int resize(Slot& S, u64 new_cap, u64 n, int from, int Wn) {
    cudaError_t e;
    u64* nk[2] = {nullptr, nullptr};
    double* nc[2] = {nullptr, nullptr};
    const u64 ntcap = 2 * new_cap;
    u64* nt = nullptr;
    u64* ns = nullptr;
    const u64 n_status = new_cap / TILE_ROWS + 2;
    auto cleanup = [&]() {
      for (int i = 0; i < 2; ++i) {
        if (nk[i]) dfree(nk[i]);
        if (nc[i]) dfree(nc[i]);
      }
      if (nt) dfree(nt);
      if (ns) dfree(ns);
    };
    for (int i = 0; i < 2; ++i) {
      if ((e = dmalloc(&nk[i], new_cap * Wn * 8)) != cudaSuccess ||
          (e = dmalloc(&nc[i], new_cap * 8)) != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "allocating term rows");
      }
    }
    if ((e = dmalloc(&nt, ntcap * 8)) != cudaSuccess || (e = dmalloc(&ns, n_status * 8)) != cudaSuccess) {
      cleanup();
      return cuda_fail(e, "allocating the hash table");
    }
    if (n && S.keys[from]) {
      cudaMemcpyAsync(nk[0], S.keys[from], n * Wn * 8, cudaMemcpyDeviceToDevice, stream);
      cudaMemcpyAsync(nc[0], S.coeffs[from], n * 8, cudaMemcpyDeviceToDevice, stream);
    }
    cudaMemsetAsync(ns, 0, n_status * 8, stream);
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) {
      cleanup();
      return cuda_fail(e, "copying rows");
    }
    S.free_rows();
    S.keys[0] = nk[0];
    S.keys[1] = nk[1];
    S.coeffs[0] = nc[0];
    S.coeffs[1] = nc[1];
    S.table = nt;
    S.status = ns;
    S.cap = new_cap;
    S.tcap = ntcap;
    S.cur = 0;
    S.W = Wn;
    return rebuild_table(S, n);
  }
  int rebuild_table(Slot& S, u64 n) {
    cudaMemsetAsync(S.table, 0xff, S.tcap * 8, stream);
    const cudaError_t e = with_words(S.W, [&](auto w) {
      return pq::launch_rebuild<decltype(w)::value>(S.keys[S.cur], n, S.table, S.tcap - 1, S.bmask, d_err, stream);
    });
    if (n) ++launches;
    if (e != cudaSuccess) return cuda_fail(e, "rebuild launch");
    return PQ_OK;
  }
  // Class-op scratch for the slot's current capacity (the family table starts
  // empty: all-ones slots, zero counts; class ops leave it empty).
  int ensure_class(Slot& S) {
    if (S.cls_cap >= S.cap && S.fam_cap >= S.tcap) {
      if (S.fam_dirty) {
        cudaMemsetAsync(S.fam_table, 0xff, S.fam_cap * 8, stream);
        cudaMemsetAsync(S.fam_aux, 0, S.fam_cap * 8, stream);
        S.fam_dirty = false;
      }
      return PQ_OK;
    }
    S.free_class();
    cudaError_t e;
    if ((e = dmalloc(&S.cls_mask, S.cap * 8)) != cudaSuccess || (e = dmalloc(&S.cls_slot, S.cap * 4)) != cudaSuccess ||
        (e = dmalloc(&S.cls_children, S.cap * 4)) != cudaSuccess ||
        (e = dmalloc(&S.fam_table, S.tcap * 8)) != cudaSuccess || (e = dmalloc(&S.fam_aux, S.tcap * 8)) != cudaSuccess) {
      S.free_class();
      return cuda_fail(e, "allocating class scratch");
    }
    cudaMemsetAsync(S.fam_table, 0xff, S.tcap * 8, stream);
    cudaMemsetAsync(S.fam_aux, 0, S.tcap * 8, stream);
    S.cls_cap = S.cap;
    S.fam_cap = S.tcap;
    S.fam_dirty = false;
    return PQ_OK;
  }
  int ensure_ops(Slot& S, size_t n_ops) {
    if (S.ops_cap >= n_ops) return PQ_OK;
    S.free_ops();
    cudaError_t e;
    if ((e = dmalloc(&S.d_ops, n_ops * sizeof(pq::OpDesc))) != cudaSuccess ||
        (e = dmalloc(&S.tickets, n_ops * 4)) != cudaSuccess ||
        (e = dmalloc(&S.hist, n_ops * 8)) != cudaSuccess || (e = dmalloc(&S.anti, n_ops * 8)) != cudaSuccess ||
        (e = dmalloc(&S.stamps, n_ops * 8)) != cudaSuccess ||
        (e = dmalloc(&S.logs, n_ops * pq::LOG_WORDS * 8)) != cudaSuccess)
      return cuda_fail(e, "allocating op arrays");
    S.ops_cap = n_ops;
    return PQ_OK;
  }
};

namespace {

template <int W>
pq::GenInfo<W> make_gen(int alg, const u64* g, int sign) {
  return pq::make_gen_info<W>(alg, g, sign);
}

// One propagation's inputs as the C ABI receives them; keys are `in_words`
// words wide (pq_words_for_units of the instance).
struct Inputs {
  const pq_run_config* cfg;
  const u64* obs_words;
  const double* obs_coeffs;
  size_t n_obs;
  const u64* gate_words;
  const double* angles;
  size_t n_gates;
  const u32* layer_off;
  size_t n_layers;
  const u64* diag;
  size_t nd;
  u64* n_terms_out;
  pq_result* res;
  int in_words;
};

// Host side of one propagation: resolved noise, the admitted observable, the
// op sequence with its gate descriptors, the Clifford frame, and how far the
// device has run it.  W is the width the device runs it at (>= in_words; the
// extra words are zero).
constexpr u32 FUSE_DEFAULT = 2;  // rotations a fused group holds unless the run says otherwise
// Slots of a hash-table bucket unless the run says otherwise: 2-slot buckets
// ran every single-run workload 0.5-1.2% faster than 4-slot ones.
constexpr u32 BUCKET_DEFAULT = 2;

struct Plan {
  const Inputs* in = nullptr;
  int W = 1, alg = 0;
  u32 n_units = 0;
  bool has_w = false, has_c = false, has_floor = false;
  u32 wcut = pq::NO_WEIGHT_CUT;
  double ccut = 0;
  u64 floor_terms = 0;
  size_t tlen = 0;
  std::vector<double> tables;
  bool layered = false, have_noise = false;
  // Plugins the host consults during the run (noise_resolver.rs:28-37,
  // termsum.rs:113-168): a truncator decides every branch and reclaim; a
  // key-reading noise model gives every row its own factor.  Either one
  // reading keys turns Clifford deferral off (engine.rs:101-103).
  const Plugin* term = nullptr;
  const Plugin* keynoise = nullptr;
  bool host_ops = false;
  bool defer = true;
  bool log = false;  // per-gate records for the verbose log (pq_run_config::log_gates)
  bool has_class = false;  // some op is a class (fuse_classes)
  // Tuning (pq_run_config / pq_batch_tuning): rotations fused into one pass,
  // rows per thread of a many-row gate tile (0 = the kernel's 4), slots per
  // table bucket.
  u32 fuse_max = FUSE_DEFAULT, tile_items = 0, bucket_slots = BUCKET_DEFAULT;
  bool fold_on_device = false;  // hk / hc hold the admitted terms unfolded (DEVICE_FOLD_MIN)
  std::vector<u64> hk;
  std::vector<double> hc;
  u64 n0 = 0;
  std::vector<pq::OpDesc> ops;
  std::vector<u64> gdesc;  // GateDesc<W> records back to back
  size_t n_gdesc = 0;
  std::vector<long> gate_op;  // latest op at or before each gate, -1 = none
  std::vector<char> gate_own;  // the gate has an op of its own (not deferred into the frame)
  std::vector<size_t> layer_op;  // first op of each layer
  Tableau frame{0, 1, 0};
  long last_op = -1;
  size_t done = 0, uploaded_ops = 0, uploaded_gdesc = 0;
  u64 rec_next = 0, rec_key_next = 0;  // adjoint recording: next free slots of the pool
  u32 rec_full = 0;
  u64 n_live = 0, peak = 0;
  double sweep_ms = 0;
  u64 sweep_launches = 0;

  // Copies key i of an input array (in_words wide) into W words.
  void widen(const u64* src, size_t i, u64* dst) const {
    for (int w = 0; w < W; ++w) dst[w] = w < in->in_words ? src[i * in->in_words + w] : 0;
  }
};

size_t gdesc_words(int W) {
  return with_words(W, [](auto w) { return sizeof(pq::GateDesc<decltype(w)::value>) / 8; });
}

// Resolves noise (noise_resolver.rs:78-131) and admits the observable with
// duplicate folding (engine.rs:104-111).
int prepare(pq_engine* E, Plan& P, const Inputs& in, int W) {
  const pq_run_config* cfg = in.cfg;
  P.in = &in;
  P.W = W;
  P.alg = (int)cfg->basis_kind;
  const int ALG = P.alg;
  P.n_units = cfg->n_units;
  P.has_w = cfg->max_weight >= 0;
  P.wcut = P.has_w ? (u32)std::min<int64_t>(cfg->max_weight, 0xfffffffe) : pq::NO_WEIGHT_CUT;
  P.has_c = cfg->has_min_coeff != 0;
  P.ccut = cfg->min_coeff;
  P.has_floor = cfg->min_terms >= 0;
  P.log = cfg->log_gates != 0;
  P.fuse_max = cfg->fuse_max ? cfg->fuse_max : FUSE_DEFAULT;
  P.tile_items = cfg->tile_items;
  P.bucket_slots = cfg->bucket_slots ? cfg->bucket_slots : BUCKET_DEFAULT;
  P.floor_terms = P.has_floor ? (u64)cfg->min_terms : 0;
  const Plugin* np = reinterpret_cast<const Plugin*>(cfg->noise_plugin);
  P.tlen = cfg->noise_table_len ? cfg->noise_table_len : (size_t)P.n_units + 1;
  P.have_noise = cfg->noise_kind != PQ_NOISE_NONE;
  if (cfg->noise_kind == PQ_NOISE_TABLE) {
    if (!cfg->noise_tables || !cfg->noise_table_len) return E->fail(PQ_ERR_INVALID, "noise table missing");
    P.tables.assign(cfg->noise_tables, cfg->noise_tables + P.tlen);
  } else if (cfg->noise_kind == PQ_NOISE_LAYERED) {
    if (!cfg->noise_tables || !cfg->noise_table_len) return E->fail(PQ_ERR_INVALID, "noise tables missing");
    P.tables.assign(cfg->noise_tables, cfg->noise_tables + P.tlen * in.n_layers);
    P.layered = true;
  } else if (cfg->noise_kind == PQ_NOISE_PLUGIN) {
    if (!np) return E->fail(PQ_ERR_INVALID, "noise plugin missing");
    P.tlen = (size_t)P.n_units + 1;
    if (np->depends & 1) P.keynoise = np;
    auto f = (NoiseFactorFn)np->fn;
    auto tab = [&](u32 layer, u32 total) {
      for (u32 w = 0; w < P.n_units + 1; ++w)
        P.tables.push_back(f(np->ctx, ALG, nullptr, 0, P.n_units, w, layer, total));
    };
    if (P.keynoise) {
      // per term, on the host at each noise op
    } else if (np->depends & 2) {
      P.layered = true;
      for (size_t l = 0; l < in.n_layers; ++l) tab((u32)l, (u32)in.n_layers);
    } else {
      tab(0, 0);
    }
  } else if (cfg->noise_kind != PQ_NOISE_NONE) {
    return E->fail(PQ_ERR_INVALID, "unknown noise kind");
  }
  P.term = reinterpret_cast<const Plugin*>(cfg->truncator);
  if (P.term && P.term->noise) return E->fail(PQ_ERR_INVALID, "the truncator handle is a noise plugin");
  if (P.keynoise && !P.keynoise->noise) return E->fail(PQ_ERR_INVALID, "the noise handle is a truncator plugin");
  P.host_ops = P.term || P.keynoise;
  P.defer = !(P.keynoise || (P.term && (P.term->depends & 1)));
  struct H {
    size_t operator()(const std::vector<u64>& v) const {
      u64 h = 0x9e3779b97f4a7c15ULL;
      for (u64 x : v) {
        h = (h ^ x) * 0xff51afd7ed558ccdULL;
        h ^= h >> 29;
      }
      return (size_t)h;
    }
  };
  std::unordered_map<std::vector<u64>, size_t, H> pos;
  std::vector<u64> k(W);
  P.fold_on_device = in.n_obs >= DEVICE_FOLD_MIN;
  for (size_t i = 0; i < in.n_obs; ++i) {
    P.widen(in.obs_words, i, k.data());
    const double c = in.obs_coeffs[i];
    if (P.term) {  // admits_initial with a term kernel: its keep alone (termsum.rs:113-160)
      const bool kd = P.term->depends & 1;
      if (!((KeepFn)P.term->fn)(P.term->ctx, ALG, kd ? k.data() : nullptr, kd ? (size_t)W : 0, P.n_units,
                                host_weight(ALG, W, k.data(), P.n_units), std::fabs(c), 0, 0))
        continue;
    } else {
      if (P.has_w && host_weight(ALG, W, k.data(), P.n_units) > P.wcut) continue;
      if (P.has_c && !(std::fabs(c) >= P.ccut)) continue;
    }
    if (P.fold_on_device) {  // folded by setup_slot on the device, in this order
      P.hk.insert(P.hk.end(), k.begin(), k.end());
      P.hc.push_back(c);
      continue;
    }
    auto it = pos.find(k);
    if (it != pos.end()) {
      P.hc[it->second] += c;
    } else {
      pos.emplace(k, P.hc.size());
      P.hk.insert(P.hk.end(), k.begin(), k.end());
      P.hc.push_back(c);
    }
  }
  P.n0 = P.hc.size();
  P.n_live = P.peak = P.n0;
  P.frame = Tableau(ALG, W, P.n_units);
  P.gate_op.assign(in.n_gates, -1);
  P.gate_own.assign(in.n_gates, 0);
  P.ops.reserve(in.n_gates + in.n_layers);
  P.gdesc.reserve(in.n_gates * gdesc_words(W));
  return PQ_OK;
}

// Sizes the slot's buffers for the plan, uploads the admitted rows and noise
// tables, rebuilds the table.
int setup_slot(pq_engine* E, Slot& S, Plan& P) {
  cudaError_t e;
  const int W = P.W;
  S.bmask = ~(u64)(P.bucket_slots - 1);
  const u64 want_cap = next_pow2(std::max<u64>(4 * P.n0, 1ULL << 16));
  if (S.W != W || S.cap < want_cap) {
    if (int rc = E->resize(S, std::max(want_cap, S.W == W ? S.cap : 0), 0, S.cur, W)) return rc;
  }
  S.cur = 0;
  if (P.n0 && P.fold_on_device) {
    // duplicates add up as the host loop would: stable sort by key, then each
    // run of equal keys summed in input order (engine.rs:104-111)
    cudaMemcpyAsync(S.keys[1], P.hk.data(), P.n0 * W * 8, cudaMemcpyHostToDevice, E->stream);
    cudaMemcpyAsync(S.coeffs[1], P.hc.data(), P.n0 * 8, cudaMemcpyHostToDevice, E->stream);
    const u64 words = pq::sort_scratch_words(P.n0, W) + (P.n0 + 1) / 2;
    if ((e = E->sort_buf.ensure(words * 8)) != cudaSuccess) return E->cuda_fail(e, "sort scratch");
    u64* scratch = E->sort_buf.at<u64>(0);
    u32* head = reinterpret_cast<u32*>(scratch + pq::sort_scratch_words(P.n0, W));
    u64 n_fold = 0;
    e = with_words(W, [&](auto w) {
      constexpr int WW = decltype(w)::value;
      cudaError_t ee = pq::sort_rows<WW>(S.keys[1], S.coeffs[1], P.n0, S.keys[0], S.coeffs[0], scratch, E->stream,
                                         &E->launches);
      if (ee == cudaSuccess)
        ee = pq::fold_sorted<WW>(S.keys[0], S.coeffs[0], P.n0, S.keys[1], S.coeffs[1], head, &n_fold, scratch,
                                 E->stream, &E->launches);
      return ee;
    });
    if (e != cudaSuccess) return E->cuda_fail(e, "folding the observable");
    S.cur = 1;
    P.n0 = P.n_live = P.peak = n_fold;
  } else if (P.n0) {
    cudaMemcpyAsync(S.keys[0], P.hk.data(), P.n0 * W * 8, cudaMemcpyHostToDevice, E->stream);
    cudaMemcpyAsync(S.coeffs[0], P.hc.data(), P.n0 * 8, cudaMemcpyHostToDevice, E->stream);
  }
  if (int rc = E->rebuild_table(S, P.n0)) return rc;
  const size_t n_ops_max = P.in->n_gates + P.in->n_layers + 1;
  if (int rc = E->ensure_ops(S, n_ops_max)) return rc;
  const size_t gbytes = std::max<size_t>(P.in->n_gates, 1) * gdesc_words(W) * 8;
  if (S.gates_bytes < gbytes) {
    if (S.d_gates) dfree(S.d_gates);
    S.d_gates = nullptr;
    S.gates_bytes = 0;
    if ((e = dmalloc(&S.d_gates, gbytes)) != cudaSuccess) return E->cuda_fail(e, "gate descriptors");
    S.gates_bytes = gbytes;
  }
  if (!P.tables.empty()) {
    if ((e = grow_pair<double>(&S.d_tables, nullptr, &S.d_tables_cap, P.tables.size())) != cudaSuccess)
      return E->cuda_fail(e, "noise tables");
    cudaMemcpyAsync(S.d_tables, P.tables.data(), P.tables.size() * 8, cudaMemcpyHostToDevice, E->stream);
  }
  if (!S.partials) {
    if ((e = dmalloc(&S.partials, sizeof(pq::ExpectPartial) * E->expect_grid)) != cudaSuccess)
      return E->cuda_fail(e, "partials");
  }
  cudaMemsetAsync(S.anti, 0, n_ops_max * 8, E->stream);
  if (P.log) cudaMemsetAsync(S.logs, 0, n_ops_max * pq::LOG_WORDS * 8, E->stream);
  if (S.epoch_base > (1u << 29)) {  // keep status tags unique: restart the epochs on a cleared array
    S.epoch_base = 1;
    cudaMemsetAsync(S.status, 0, (S.cap / TILE_ROWS + 2) * 8, E->stream);
  }
  return PQ_OK;
}

// Appends the op sequence (engine.rs:117-205, partitioned_termsum.rs:282-350).
// need_n(&n) is called when the Clifford deferral decision depends on the
// live count (TermBudget with a weight cut); it must run the ops built so far
// and report the live count.
template <class NeedN>
int build_ops(Plan& P, NeedN need_n) {
  const Inputs& in = *P.in;
  const int W = P.W, ALG = P.alg;
  std::vector<u64> g(W), gc(W);
  P.gdesc.reserve(P.gdesc.size() + in.n_gates * gdesc_words(W));
  P.ops.reserve(P.ops.size() + in.n_gates + in.n_layers);
  for (size_t l = 0; l < in.n_layers; ++l) {
    P.layer_op.push_back(P.ops.size());
    if (P.have_noise) {
      pq::OpDesc od;
      od.kind = (P.has_w || P.has_c || P.term) ? pq::OP_NOISE_COMPACT : pq::OP_NOISE_SCALE;  // partitioned_termsum.rs:585-587
      od.idx = P.layered ? (u32)l : 0u;
      P.ops.push_back(od);
      P.last_op = (long)P.ops.size() - 1;
    }
    for (u32 gi = in.layer_off[l]; gi < in.layer_off[l + 1]; ++gi) {
      P.widen(in.gate_words, gi, g.data());
      const double ang = in.angles[gi];
      if (P.defer && std::fabs(std::cos(ang)) < EPS_CLASSIFY) {  // Clifford: defer into the frame when allowed
        bool eff_w = P.has_w;
        const bool cw = Tableau::rotation_changes_weight(ALG, W, P.n_units, g.data());
        if (P.has_w && cw && P.has_floor) {  // the effective cutoff depends on the live count here
          u64 n = 0;
          if (int rc = need_n(&n)) return rc;
          if (n < P.floor_terms) eff_w = false;
        }
        if (!eff_w || !cw) {
          P.frame.compose_rotation(g.data(), ang);
          P.gate_op[gi] = P.last_op;
          continue;
        }
      }
      const int sign = P.frame.conjugate_generator(g.data(), gc.data());
      const double sn = std::sin(ang), cs = std::cos(ang);
      with_words(W, [&](auto w) {
        constexpr int WW = decltype(w)::value;
        pq::GateDesc<WW> gd;
        gd.g = make_gen<WW>(ALG, gc.data(), sign);
        gd.sn = sn;
        gd.cs = cs;
        gd.pivot = 0;
        gd.pad_ = 0;
        const size_t off = P.gdesc.size();
        P.gdesc.resize(off + sizeof gd / 8);
        std::memcpy(&P.gdesc[off], &gd, sizeof gd);
        return 0;
      });
      pq::OpDesc od;
      od.kind = std::fabs(sn) < EPS_CLASSIFY ? pq::OP_PHASE : pq::OP_GATE;
      od.idx = (u32)P.n_gdesc++;
      P.ops.push_back(od);
      P.last_op = (long)P.ops.size() - 1;
      P.gate_op[gi] = P.last_op;
      P.gate_own[gi] = 1;
    }
  }
  P.layer_op.push_back(P.ops.size());
  return PQ_OK;
}

// Marks runs of CLASS_MIN to CLASS_MAX consecutive Pauli rotation ops whose
// generators act on pairwise disjoint qubits as classes (OP_CLASS head,
// OP_GATE_TAIL for the rest): the sweep runs each in one op (class_op), every
// family of keys through all its rotations at once.  Each generator's pivot
// is its lowest key bit, which no other generator of the class has.  Only
// where the family dimension of every live row is bounded by CLASS_KMAX: a
// weight cut of at most CLASS_KMAX bounds every row's weight, and a row
// anticommutes with at most one generator per qubit of its support.  Not with
// a TermBudget floor (its lossless switch reads the live count between
// rotations), host decisions, the verbose log (per-rotation times) or the
// adjoint's recording (which does not call this).  Only runs of Clifford
// rotations (|cos| < 1e-9, kept out of the frame because they change weight
// under a weight cut): their sin branches carry the whole coefficient, so a
// family stays small (one new member per step) and runs in one thread; a run
// of generic angles makes families of up to 2^k members, which a single warp
// runs slower than pair-fused ops over all rows (measured with generic runs
// of 8 or more rotations as classes: kicked Ising 10x10 x 20 steps 104 ms
// against 24.8 ms, the TFIM chain 5.5 ms against 1.8 ms).
constexpr size_t CLASS_MIN = 4;
void fuse_classes(Plan& P) {
  if (P.alg != 0 || P.W > 4 || P.has_floor || P.host_ops || P.log) return;
  if (!P.has_w || P.wcut > pq::CLASS_KMAX) return;
  const size_t gw = gdesc_words(P.W);
  const int W = P.W;
  auto gen = [&](size_t op) { return &P.gdesc[P.ops[op].idx * gw]; };
  auto support = [&](const u64* g, int w) { return (g[w] | (g[w] >> 1)) & EVEN; };
  auto clifford = [&](size_t op) {
    return with_words(W, [&](auto ww) {
      constexpr int WW = decltype(ww)::value;
      pq::GateDesc<WW> gd;
      std::memcpy(&gd, gen(op), sizeof gd);
      return std::fabs(gd.cs) < EPS_CLASSIFY;
    });
  };
  for (size_t i = 0; i < P.ops.size(); ++i) {
    if (P.ops[i].kind != pq::OP_GATE) continue;
    std::vector<u64> used(W, 0);
    size_t n = 0;
    while (n < pq::CLASS_MAX && i + n < P.ops.size() && P.ops[i + n].kind == pq::OP_GATE &&
           P.ops[i + n].idx == P.ops[i].idx + n && clifford(i + n)) {
      const u64* g = gen(i + n);
      bool ok = false, clash = false;
      for (int w = 0; w < W; ++w) {
        ok |= g[w] != 0;
        clash |= (support(g, w) & used[w]) != 0;
      }
      if (!ok || clash) break;
      for (int w = 0; w < W; ++w) used[w] |= support(g, w);
      ++n;
    }
    if (n < CLASS_MIN) continue;
    for (size_t m = 0; m < n; ++m) {  // pivots: each generator's lowest bit
      const u64* g = gen(i + m);
      u32 piv = 0;
      for (int w = 0; w < W; ++w)
        if (g[w]) {
          piv = (u32)(64 * w + __builtin_ctzll(g[w]));
          break;
        }
      with_words(W, [&](auto ww) {
        constexpr int WW = decltype(ww)::value;
        pq::GateDesc<WW> gd;
        u64* at = &P.gdesc[P.ops[i + m].idx * gw];
        std::memcpy(&gd, at, sizeof gd);
        gd.pivot = piv;
        std::memcpy(at, &gd, sizeof gd);
        return 0;
      });
    }
    P.ops[i].kind = pq::class_kind((u32)n);
    for (size_t m = 1; m < n; ++m) P.ops[i + m].kind = pq::OP_GATE_TAIL;
    P.has_class = true;
    i += n - 1;
  }
}

// Marks runs of up to fuse_max (1 or 2, default 2) consecutive rotation ops
// whose (frame-conjugated) generators pairwise commute and are independent
// (no subset multiplies to the identity, so a family's members are distinct)
// as fused groups: a head OP_GATE2 and an OP_GATE_TAIL op.  The sweep runs a
// pair in one pass (gate2_tiles) while every block has at most a few tiles,
// else one rotation after the other.  Pairs only: one-pass kernels for 3 and
// 4 rotations were slower on every workload measured -- first with families
// of 8 and 16 keys in registers (kicked Ising 10x10 x 20 steps 46.6 and 52.4
// ms against 42.0 ms), then with each row's family over only the rotations it
// anticommutes with (28.4 ms for groups of 4 against 23.4 ms for pairs, the
// RX layers 19.2 against 14.4 ms): their per-family work outweighs the
// barriers they save.  Not with a TermBudget floor: its lossless switch reads
// the live count between rotations; not when the host decides branches; and
// the adjoint's runs do not fuse (each rotation needs its own record).
void fuse_groups(Plan& P) {
  const size_t FUSE_MAX = std::min<size_t>(P.fuse_max, pq::GROUP_MAX);
  if (P.has_floor || P.host_ops || P.log) return;
  const size_t gw = gdesc_words(P.W);
  const int W = P.W;
  auto gen = [&](size_t op) { return &P.gdesc[P.ops[op].idx * gw]; };  // GateDesc starts with the generator
  for (size_t i = 0; i < P.ops.size(); ++i) {
    if (P.ops[i].kind != pq::OP_GATE) continue;
    // the XORs of every subset of the group so far (span over GF(2))
    std::vector<std::vector<u64>> span{std::vector<u64>(W, 0), std::vector<u64>(gen(i), gen(i) + W)};
    size_t n = 1;
    while (n < FUSE_MAX && i + n < P.ops.size() && P.ops[i + n].kind == pq::OP_GATE &&
           P.ops[i + n].idx == P.ops[i].idx + n) {
      const u64* g = gen(i + n);
      bool ok = true;
      for (size_t m = 0; m < n && ok; ++m) ok = !host_anticommutes(P.alg, W, gen(i + m), g);
      for (const auto& v : span) {  // independent: g is not the product of any subset
        if (!ok) break;
        ok = !std::equal(v.begin(), v.end(), g);
      }
      if (!ok) break;
      const size_t before = span.size();
      for (size_t k = 0; k < before; ++k) {
        std::vector<u64> v = span[k];
        for (int w = 0; w < W; ++w) v[w] ^= g[w];
        span.push_back(v);
      }
      ++n;
    }
    if (n < 2) continue;
    P.ops[i].kind = n == 2 ? pq::OP_GATE2 : (n == 3 ? pq::OP_GATE3 : pq::OP_GATE4);
    for (size_t m = 1; m < n; ++m) P.ops[i + m].kind = pq::OP_GATE_TAIL;
    i += n - 1;
  }
}

// Enqueues the upload of the ops and gate descriptors not yet on the device.
void upload_ops(pq_engine* E, Slot& S, Plan& P) {
  if (P.ops.size() > P.uploaded_ops) {
    cudaMemcpyAsync(S.d_ops + P.uploaded_ops, P.ops.data() + P.uploaded_ops,
                    (P.ops.size() - P.uploaded_ops) * sizeof(pq::OpDesc), cudaMemcpyHostToDevice, E->stream);
    P.uploaded_ops = P.ops.size();
  }
  if (P.gdesc.size() > P.uploaded_gdesc) {
    cudaMemcpyAsync(reinterpret_cast<u64*>(S.d_gates) + P.uploaded_gdesc, P.gdesc.data() + P.uploaded_gdesc,
                    (P.gdesc.size() - P.uploaded_gdesc) * 8, cudaMemcpyHostToDevice, E->stream);
    P.uploaded_gdesc = P.gdesc.size();
  }
}

// Device arrays of the adjoint's recording (see SweepArgs::rec_idx).
struct Recording {
  u32* idx = nullptr;
  double* coef = nullptr;
  u64* keys = nullptr;
  u64* off = nullptr;      // written by the sweep, per op
  u64* key_off = nullptr;
  u64 cap = 0, key_cap = 0;  // elements of idx / coef, rows of keys
};

// Per-row decisions made on the host for one op (device pointers, or null).
struct HostOps {
  const unsigned char* state = nullptr;
  const double* factor = nullptr;
  const unsigned char* keep = nullptr;
};

pq::SweepArgs sweep_args(Slot& S, const Plan& P, pq::SweepState* st, u32 blk_begin, u32 blk_count,
                         size_t op_limit = (size_t)-1, const Recording* rec = nullptr,
                         const HostOps* host = nullptr) {
  pq::SweepArgs a{};
  a.ops = S.d_ops;
  a.gates = S.d_gates;
  a.n_gdesc = (u32)(P.gdesc.size() / gdesc_words(P.W));
  a.tables = S.d_tables;
  a.table_len = (u32)P.tlen;
  a.n_units = P.n_units;
  a.n_words = (u32)P.W;
  a.op_begin = (u32)P.done;
  a.op_end = (u32)std::min(op_limit, P.ops.size());
  if (host) {
    a.host_state = host->state;
    a.host_factor = host->factor;
    a.host_keep = host->keep;
  }
  if (rec) {
    a.rec_idx = rec->idx;
    a.rec_coef = rec->coef;
    a.rec_keys = rec->keys;
    a.rec_off = rec->off;
    a.rec_key_off = rec->key_off;
    a.rec_cap = rec->cap;
    a.rec_key_cap = rec->key_cap;
  }
  a.cur0 = (u32)S.cur;
  a.epoch_base = S.epoch_base;
  a.max_weight = P.wcut;
  a.has_min_coeff = P.has_c;
  a.min_coeff = P.ccut;
  a.min_terms = P.floor_terms;
  for (int i = 0; i < 2; ++i) {
    a.keys[i] = S.keys[i];
    a.coeffs[i] = S.coeffs[i];
  }
  a.table = S.table;
  a.table_mask = S.tcap - 1;
  a.table_bmask = S.bmask;
  a.tile_items = P.tile_items;
  a.cap = S.cap;
  a.status = S.status;
  a.tickets = S.tickets;
  a.hist = S.hist;
  a.anti = S.anti;
  a.stamps = S.stamps;
  a.log = P.log ? S.logs : nullptr;
  if (P.has_class) {
    a.cls_mask = S.cls_mask;
    a.cls_slot = S.cls_slot;
    a.cls_children = S.cls_children;
    a.fam_table = S.fam_table;
    a.fam_aux = S.fam_aux;
  }
  a.st = st;
  a.blk_begin = blk_begin;
  a.blk_count = blk_count;
  return a;
}

pq::SweepState fresh_state(const pq_engine* E, const Plan& P) {
  pq::SweepState s{};
  E->init_waits(s);
  s.n[P.done & 1] = P.n_live;
  s.peak = P.peak;
  s.halt = pq::NOT_HALTED;
  s.rec_next = P.rec_next;
  s.rec_key_next = P.rec_key_next;
  s.rec_full = P.rec_full;
  return s;
}

// Reads a plan's sweep state after a launch; on a capacity halt grows its rows
// (the gate at `done` needs 2 N rows) so that the next launch resumes there.
int absorb_state(pq_engine* E, Slot& S, Plan& P, const pq::SweepState& h) {
  // The launch tagged its tile statuses with epochs from epoch_base; the next
  // launch must use fresh ones even when this one failed part way, or it
  // could read this launch's statuses as its own.
  S.epoch_base += (u32)P.ops.size() + 1;
  if (h.error) S.fam_dirty = true;
  if (h.error & pq::ERR_BARRIER_TIMEOUT)
    return E->fail(PQ_ERR_DEVICE_TIMEOUT, "a grid barrier wait expired on the device");
  if (h.error & pq::ERR_LOOKBACK_TIMEOUT)
    return E->fail(PQ_ERR_DEVICE_TIMEOUT, "a tile's look-back wait expired on the device");
  if (h.error) return E->fail(PQ_ERR_CUDA, "device reported error bits " + std::to_string(h.error));
  S.cur = (int)h.cur;
  P.done = h.end_op;
  P.n_live = h.n[P.done & 1];
  P.peak = std::max(P.peak, h.peak);
  P.rec_next = h.rec_next;
  P.rec_key_next = h.rec_key_next;
  P.rec_full = h.rec_full;
  ++P.sweep_launches;
  if (h.halt != pq::NOT_HALTED && !h.grid_stop) {
    // a class op reports the rows it would leave (need_rows); the next op
    // may double them
    u64 ncap = next_pow2(std::max<u64>(std::max<u64>(4 * P.n_live, 2 * std::min(S.cap, E->row_ceiling())),
                                       2 * h.need_rows));
    if (ncap > E->row_ceiling()) ncap = E->row_ceiling();
    if (2 * P.n_live > ncap || h.need_rows > ncap)
      return E->fail(PQ_ERR_CEILING, "term index ceiling reached: " + std::to_string(2 * P.n_live) +
                                         " rows would exceed the engine's capacity");
    if (ncap <= S.cap) return PQ_OK;  // the ceiling was below the buffers: they already hold ncap rows
    int rc = E->resize(S, ncap, P.n_live, S.cur, P.W);
    if (rc == PQ_ERR_OOM) rc = E->resize(S, next_pow2(2 * P.n_live), P.n_live, S.cur, P.W);
    if (rc) return rc;
  }
  return PQ_OK;
}

// Grid of one sweep launch.  With blocks_per_sm 0 (the default) it follows
// the live count at the launch: one block per SM while every row has a thread
// of its own, two per SM up to 2^20 rows, else `max_grid`; and for 1- and
// 2-word keys from 2^24 rows on, the sweep built for six resident blocks per
// SM (sweep_kernel_occ).  A grid below the largest carries the row count it
// is chosen for (SweepArgs::grid_rows); the sweep stops before an op that
// outgrows it and the next launch takes the next size.  Fewer blocks make the
// grid barrier between ops cheaper (one block per SM took TFIM from 1.95 to
// 1.74 ms), more blocks keep more rows in flight (the 24-site Majorana run
// needs them: 35 ms at the largest grid, 76 ms at one block per SM).
struct GridChoice {
  int grid;
  u64 rows;   // 0: no limit
  int build;  // pq::SweepBuild of the kernel to launch
};
constexpr u64 OCC_ROWS = 1ULL << 24;
GridChoice choose_grid(const Plan& P, const Inputs& in, int max_grid) {
  if (in.cfg->blocks_per_sm != 0) return {max_grid, 0, pq::SWEEP_DEFAULT};
  const auto tier = [&](int bps, int build) {
    return with_words(P.W, [&](auto w) {
      constexpr int WW = decltype(w)::value;
      return P.alg == 0 ? pq::sweep_grid<WW, 0>(bps, build) : pq::sweep_grid<WW, 1>(bps, build);
    });
  };
  // the one- and two-block tiers run the two-block build (keys of at most 4 words)
  const int small = P.W <= 4 ? pq::SWEEP_TWO : pq::SWEEP_DEFAULT;
  const int g1 = tier(1, small), g2 = tier(2, small);
  const u64 r1 = (u64)g1 * 256, r2 = 1ULL << 20;
  if (g1 < max_grid && P.n_live <= r1) return {g1, r1, small};
  if (g2 < max_grid && P.n_live <= r2) return {g2, r2, small};
  if (P.W > 2) return {max_grid, 0, pq::SWEEP_DEFAULT};
  if (P.n_live <= OCC_ROWS) return {max_grid, OCC_ROWS, pq::SWEEP_DEFAULT};
  return {tier(0, pq::SWEEP_SIX), 0, pq::SWEEP_SIX};
}

// Runs every built op of one plan, relaunching after capacity growth and when
// the live count outgrows the launch's grid (choose_grid).
int execute_launches(pq_engine* E, Slot& S, Plan& P, int grid, bool* began, size_t op_limit,
                     const Recording* rec, const HostOps* host) {
  cudaError_t e;
  upload_ops(E, S, P);
  const size_t end = std::min(op_limit, P.ops.size());
  const int max_grid = grid;
  while (P.done < end) {
    if (P.has_class)
      if (int rc = E->ensure_class(S)) return rc;
    const GridChoice gc = choose_grid(P, *P.in, max_grid);
    grid = gc.grid;
    E->h_states[0] = fresh_state(E, P);
    cudaMemcpyAsync(E->d_states, E->h_states, sizeof(pq::SweepState), cudaMemcpyHostToDevice, E->stream);
    cudaMemsetAsync(S.tickets + P.done, 0, (end - P.done) * 4, E->stream);
    pq::SweepArgs a = sweep_args(S, P, E->d_states, 0, (u32)grid, end, rec, host);
    a.grid_rows = gc.rows;
    E->limit_args(a);
    if (!*began) {  // device time starts at the first sweep
      cudaEventRecord(E->ev_begin, E->stream);
      *began = true;
    }
    cudaEventRecord(E->ev_l0, E->stream);
    e = with_words(P.W, [&](auto w) {
      constexpr int WW = decltype(w)::value;
      return P.alg == 0 ? pq::launch_sweep<WW, 0>(a, grid, E->stream, gc.build)
                        : pq::launch_sweep<WW, 1>(a, grid, E->stream, gc.build);
    });
    if (e != cudaSuccess) return E->cuda_fail(e, "sweep launch");
    cudaEventRecord(E->ev_l1, E->stream);
    ++E->launches;
    cudaMemcpyAsync(E->h_states, E->d_states, sizeof(pq::SweepState), cudaMemcpyDeviceToHost, E->stream);
    if ((e = cudaStreamSynchronize(E->stream)) != cudaSuccess) return E->cuda_fail(e, "sweep");
    float ms = 0;
    cudaEventElapsedTime(&ms, E->ev_l0, E->ev_l1);
    P.sweep_ms += ms;
    if (int rc = absorb_state(E, S, P, E->h_states[0])) return rc;
  }
  return PQ_OK;
}

// True if op k needs decisions from a plugin on the host: every rotation when
// a truncator is set (its keep decides each branch), every noise op when the
// noise model reads keys or a truncator decides the reclaim.
bool needs_host(const Plan& P, size_t k) {
  const u32 kind = P.ops[k].kind;
  if (kind == pq::OP_GATE) return P.term != nullptr;
  if (kind == pq::OP_NOISE_SCALE || kind == pq::OP_NOISE_COMPACT) return P.keynoise || P.term;
  return false;
}

u32 layer_of(const Plan& P, size_t k) {
  const auto it = std::upper_bound(P.layer_op.begin(), P.layer_op.end(), k);
  return (u32)(it - P.layer_op.begin()) - 1;
}

// Reads the live rows back and asks the plugins for op k's decisions, exactly
// where the reference asks them: a truncator's scalar keep for every branch
// (termsum.rs:701-751, with the branch's coefficient and child key), a
// key-reading noise model's factor for every row (factor_batch in chunks of
// 1024 when the plugin has it, termsum.rs:340-371), and the truncator's
// keep_batch on the damped rows for the reclaim (termsum.rs:387-447).  A
// rotation under the TermBudget floor runs with no truncation at all.
int host_decide(pq_engine* E, Slot& S, Plan& P, size_t k, HostOps* ho) {
  *ho = HostOps{};
  const int W = P.W, ALG = P.alg;
  const u64 N = P.n_live;
  const u32 kind = P.ops[k].kind;
  if (kind == pq::OP_GATE && P.has_floor && N < P.floor_terms) return PQ_OK;
  if (N == 0) return PQ_OK;
  cudaError_t e;
  if (S.host_cap < N) {
    for (void* p : {(void*)S.host_state, (void*)S.host_factor, (void*)S.host_keep})
      if (p) dfree(p);
    S.host_state = nullptr;
    S.host_factor = nullptr;
    S.host_keep = nullptr;
    S.host_cap = 0;
    const size_t cap = std::max<size_t>(N, S.cap);
    if ((e = dmalloc(&S.host_state, cap)) != cudaSuccess || (e = dmalloc(&S.host_factor, cap * 8)) != cudaSuccess ||
        (e = dmalloc(&S.host_keep, cap)) != cudaSuccess)
      return E->cuda_fail(e, "host decision buffers");
    S.host_cap = cap;
  }
  std::vector<u64> keys(N * W);
  std::vector<double> co(N);
  cudaMemcpyAsync(keys.data(), S.keys[S.cur], N * W * 8, cudaMemcpyDeviceToHost, E->stream);
  cudaMemcpyAsync(co.data(), S.coeffs[S.cur], N * 8, cudaMemcpyDeviceToHost, E->stream);
  if ((e = cudaStreamSynchronize(E->stream)) != cudaSuccess) return E->cuda_fail(e, "reading rows back");
  const u32 layer = layer_of(P, k), n_layers = (u32)P.in->n_layers;
  if (kind == pq::OP_GATE) {
    const Plugin* t = P.term;
    const bool kd = t->depends & 1;
    std::vector<u64> gen(W), child(W);
    double sign = 1.0, sn = 0.0;
    with_words(W, [&](auto w) {
      constexpr int WW = decltype(w)::value;
      pq::GateDesc<WW> gd;
      std::memcpy(&gd, &P.gdesc[P.ops[k].idx * gdesc_words(W)], sizeof gd);
      for (int i = 0; i < WW; ++i) gen[i] = gd.g.gen[i];
      sign = gd.g.sign;
      sn = gd.sn;
      return 0;
    });
    std::vector<unsigned char> st(N, 0);
    for (u64 r = 0; r < N; ++r) {
      const u64* kr = &keys[r * W];
      if (!host_anticommutes(ALG, W, gen.data(), kr)) continue;
      for (int i = 0; i < W; ++i) child[i] = kr[i] ^ gen[i];
      const int p = host_product_exp(ALG, W, gen.data(), kr);
      const double ni = p == 1 ? -sign : (p == 3 ? sign : 0.0);
      const double b = (co[r] * sn) * ni;
      const bool keep = ((KeepFn)t->fn)(t->ctx, ALG, kd ? child.data() : nullptr, kd ? (size_t)W : 0, P.n_units,
                                        host_weight(ALG, W, child.data(), P.n_units), std::fabs(b), layer,
                                        n_layers) != 0;
      st[r] = keep ? 0 : 1;  // S_EMIT : S_HELD
    }
    cudaMemcpyAsync(S.host_state, st.data(), N, cudaMemcpyHostToDevice, E->stream);
    ho->state = S.host_state;
  } else {
    std::vector<u32> wts(N);
    for (u64 r = 0; r < N; ++r) wts[r] = host_weight(ALG, W, &keys[r * W], P.n_units);
    std::vector<double> f(N);
    if (P.keynoise) {
      const Plugin* np = P.keynoise;
      const bool kd = np->depends & 1;
      for (u64 s0 = 0; s0 < N; s0 += KERNEL_BATCH) {
        const size_t len = (size_t)std::min<u64>(KERNEL_BATCH, N - s0);
        bool done = false;
        if (np->batch_fn)
          done = ((NoiseBatchFn)np->batch_fn)(np->ctx, ALG, kd ? &keys[s0 * W] : nullptr, kd ? (size_t)W : 0,
                                              P.n_units, &wts[s0], layer, n_layers, &f[s0], len) == 0;
        if (!done)
          for (size_t j = 0; j < len; ++j)
            f[s0 + j] = ((NoiseFactorFn)np->fn)(np->ctx, ALG, kd ? &keys[(s0 + j) * W] : nullptr,
                                                kd ? (size_t)W : 0, P.n_units, wts[s0 + j], layer, n_layers);
      }
      cudaMemcpyAsync(S.host_factor, f.data(), N * 8, cudaMemcpyHostToDevice, E->stream);
      ho->factor = S.host_factor;
    } else {
      const double* tab = P.tables.data() + (P.layered ? (size_t)P.ops[k].idx * P.tlen : 0);
      for (u64 r = 0; r < N; ++r) f[r] = tab[std::min<size_t>(wts[r], P.tlen - 1)];
    }
    if (P.term && kind == pq::OP_NOISE_COMPACT) {
      const Plugin* t = P.term;
      const bool kd = t->depends & 1;
      std::vector<double> mags(N);
      for (u64 r = 0; r < N; ++r) mags[r] = std::fabs(co[r] * f[r]);
      std::vector<unsigned char> keep(N);
      for (u64 s0 = 0; s0 < N; s0 += KERNEL_BATCH) {
        const size_t len = (size_t)std::min<u64>(KERNEL_BATCH, N - s0);
        bool done = false;
        if (t->batch_fn)
          done = ((KeepBatchFn)t->batch_fn)(t->ctx, ALG, kd ? &keys[s0 * W] : nullptr, kd ? (size_t)W : 0,
                                            P.n_units, &wts[s0], &mags[s0], layer, n_layers, &keep[s0], len) == 0;
        if (done) {
          for (size_t j = 0; j < len; ++j) keep[s0 + j] = keep[s0 + j] != 0;
        } else {
          for (size_t j = 0; j < len; ++j)
            keep[s0 + j] = ((KeepFn)t->fn)(t->ctx, ALG, kd ? &keys[(s0 + j) * W] : nullptr, kd ? (size_t)W : 0,
                                           P.n_units, wts[s0 + j], mags[s0 + j], layer, n_layers) != 0;
        }
      }
      cudaMemcpyAsync(S.host_keep, keep.data(), N, cudaMemcpyHostToDevice, E->stream);
      ho->keep = S.host_keep;
    }
  }
  return PQ_OK;
}

// Runs ops up to op_limit: whole stretches in one launch, and every op that
// needs a plugin's decisions on its own, after host_decide.
int execute_single(pq_engine* E, Slot& S, Plan& P, int grid, bool* began, size_t op_limit = (size_t)-1,
                   const Recording* rec = nullptr) {
  if (!P.host_ops) return execute_launches(E, S, P, grid, began, op_limit, rec, nullptr);
  const size_t end = std::min(op_limit, P.ops.size());
  while (P.done < end) {
    size_t h = P.done;
    while (h < end && !needs_host(P, h)) ++h;
    if (h > P.done) {
      if (int rc = execute_launches(E, S, P, grid, began, h, rec, nullptr)) return rc;
      continue;
    }
    HostOps ho;
    if (int rc = host_decide(E, S, P, h, &ho)) return rc;
    if (int rc = execute_launches(E, S, P, grid, began, h + 1, rec, &ho)) return rc;
  }
  return PQ_OK;
}

// Arguments of the readout kernels: the basis state in key layout and the
// frame (uploaded by finalize).
pq::ExpectArgs expect_args(const Slot& S, const Plan& P) {
  const Inputs& in = *P.in;
  pq::ExpectArgs xa{};
  if (in.diag) {
    for (u32 u = 0; u < P.n_units; ++u) {
      const u64 bit = (u / 64 < in.nd) ? (in.diag[u / 64] >> (u % 64)) & 1 : 0;
      if (!bit) continue;
      const u32 pos = P.alg == 0 ? 2 * u + 1 : 2 * u;
      if (pos / 64 < (u32)P.W) xa.state[pos / 64] |= 1ULL << (pos % 64);
    }
  }
  xa.n_units = P.n_units;
  xa.has_min_coeff = P.has_c;
  xa.min_coeff = P.ccut;
  xa.frame_images = P.frame.identity ? nullptr : S.frame_img;
  xa.frame_signs = P.frame.identity ? nullptr : S.frame_sgn;
  xa.frame_rows = (u32)P.frame.rows;
  return xa;
}

// Enqueues the expectation value and the final-term readout of one plan.
int finalize(pq_engine* E, Slot& S, Plan& P, std::vector<pq::ExpectPartial>* parts) {
  cudaError_t e;
  const Inputs& in = *P.in;
  const int W = P.W, ALG = P.alg;
  const u64 n_fin = P.n_live;
  if (!P.frame.identity) {
    const size_t ni = P.frame.rd_img.size(), ns = P.frame.rd_sign.size();
    if (S.frame_cap < ni) {
      if (S.frame_img) dfree(S.frame_img);
      if (S.frame_sgn) dfree(S.frame_sgn);
      S.frame_img = nullptr;
      S.frame_sgn = nullptr;
      S.frame_cap = 0;
      if ((e = dmalloc(&S.frame_img, ni * 8)) != cudaSuccess) return E->cuda_fail(e, "frame");
      if ((e = dmalloc(&S.frame_sgn, ni * sizeof(int))) != cudaSuccess) return E->cuda_fail(e, "frame");
      S.frame_cap = ni;
    }
    cudaMemcpyAsync(S.frame_img, P.frame.rd_img.data(), ni * 8, cudaMemcpyHostToDevice, E->stream);
    cudaMemcpyAsync(S.frame_sgn, P.frame.rd_sign.data(), ns * sizeof(int), cudaMemcpyHostToDevice, E->stream);
  }
  const u64* d_img = P.frame.identity ? nullptr : S.frame_img;
  const int* d_sgn = P.frame.identity ? nullptr : S.frame_sgn;
  parts->clear();
  if (in.diag || P.has_c) {
    const pq::ExpectArgs xa = expect_args(S, P);
    ++E->launches;
    e = with_words(W, [&](auto w) {
      constexpr int WW = decltype(w)::value;
      return ALG == 0 ? pq::launch_expect<WW, 0>(xa, S.keys[S.cur], S.coeffs[S.cur], n_fin, S.partials,
                                                  E->expect_grid, E->stream)
                      : pq::launch_expect<WW, 1>(xa, S.keys[S.cur], S.coeffs[S.cur], n_fin, S.partials,
                                                  E->expect_grid, E->stream);
    });
    if (e != cudaSuccess) return E->cuda_fail(e, "expectation launch");
    parts->resize(E->expect_grid);
    cudaMemcpyAsync(parts->data(), S.partials, parts->size() * sizeof(pq::ExpectPartial), cudaMemcpyDeviceToHost,
                    E->stream);
  }
  S.out_keys.clear();
  S.out_coeffs.clear();
  S.out_words = in.in_words;
  if (in.cfg->want_terms && n_fin) {
    S.out_keys.resize(n_fin * W);
    S.out_coeffs.resize(n_fin);
    int src = S.cur;
    if (!P.frame.identity) {  // the alternate buffer is free after the sweep: conjugate into it
      src = S.cur ^ 1;
      ++E->launches;
      with_words(W, [&](auto w) {
        pq::launch_conjugate<decltype(w)::value>(S.keys[S.cur], S.coeffs[S.cur], n_fin, d_img, d_sgn,
                                                 (u32)P.frame.rows, ALG, S.keys[src], S.coeffs[src], E->stream);
        return 0;
      });
    }
    const u64* out_k = S.keys[src];
    const double* out_c = S.coeffs[src];
    if (in.cfg->want_terms == 2) {  // in key order: the radix sort into the engine's sort buffer
      const u64 sw = pq::sort_scratch_words(n_fin, W);
      if ((e = E->sort_buf.ensure((sw + n_fin * (u64)(W + 1)) * 8)) != cudaSuccess)
        return E->cuda_fail(e, "sort scratch");
      u64* scratch = E->sort_buf.at<u64>(0);
      u64* sk = scratch + sw;
      double* sc = reinterpret_cast<double*>(sk + n_fin * W);
      e = with_words(W, [&](auto w) {
        return pq::sort_rows<decltype(w)::value>(out_k, out_c, n_fin, sk, sc, scratch, E->stream, &E->launches);
      });
      if (e != cudaSuccess) return E->cuda_fail(e, "sorting the terms");
      out_k = sk;
      out_c = sc;
    }
    cudaMemcpyAsync(S.out_keys.data(), out_k, n_fin * W * 8, cudaMemcpyDeviceToHost, E->stream);
    cudaMemcpyAsync(S.out_coeffs.data(), out_c, n_fin * 8, cudaMemcpyDeviceToHost, E->stream);
  }
  return PQ_OK;
}

// Host half of the result, once the stream has drained: the double-double
// sum of the partials, per-gate live counts and the per-kind totals (inputs
// of the algorithmic-bytes roofline, and the device-clock split of the sweep).
int finish(pq_engine* E, Slot& S, Plan& P, const std::vector<pq::ExpectPartial>& parts) {
  const Inputs& in = *P.in;
  pq_result* res = in.res;
  if (!parts.empty()) {
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
    if (in.diag) res->expectation_value = hi + lo;
    res->terms_below_cutoff = P.has_c ? below : 0;
  }
  if (S.out_words < P.W && !S.out_coeffs.empty()) {  // drop the zero words the device width added
    const size_t n = S.out_coeffs.size();
    for (size_t i = 0; i < n; ++i)
      for (int w = 0; w < S.out_words; ++w) S.out_keys[i * S.out_words + w] = S.out_keys[i * P.W + w];
    S.out_keys.resize(n * S.out_words);
  }
  const size_t no = P.ops.size();
  std::vector<u64> hist(no), anti(no), stamps(no);
  if (no) {
    cudaMemcpyAsync(hist.data(), S.hist, no * 8, cudaMemcpyDeviceToHost, E->stream);
    cudaMemcpyAsync(anti.data(), S.anti, no * 8, cudaMemcpyDeviceToHost, E->stream);
    cudaMemcpyAsync(stamps.data(), S.stamps, no * 8, cudaMemcpyDeviceToHost, E->stream);
    if (cudaError_t e = cudaStreamSynchronize(E->stream)) return E->cuda_fail(e, "op statistics");
  }
  if (in.n_terms_out)
    for (size_t g = 0; g < in.n_gates; ++g) in.n_terms_out[g] = P.gate_op[g] >= 0 ? hist[P.gate_op[g]] : P.n0;
  S.gate_log.clear();
  {  // crates/pauli/src/engine.rs:166-193 (GateRecord), one per gate in Heisenberg order
    std::vector<u64> lg(P.log ? no * pq::LOG_WORDS : 0);
    if (no && P.log) cudaMemcpy(lg.data(), S.logs, lg.size() * 8, cudaMemcpyDeviceToHost);
    S.gate_log.resize(in.n_gates);
    for (size_t l = 0; l < in.n_layers; ++l)
      for (u32 g = in.layer_off[l]; g < in.layer_off[l + 1]; ++g) {
        pq_gate_record& rcd = S.gate_log[g];
        rcd = pq_gate_record{};
        rcd.layer_idx = (u32)l;
        const long op = P.gate_own[g] ? P.gate_op[g] : -1;
        rcd.op = (int32_t)op;
        const u64 after = P.gate_op[g] >= 0 ? hist[P.gate_op[g]] : P.n0;
        rcd.terms_after = after;
        rcd.terms_before = op > 0 ? hist[op - 1] : (op == 0 ? P.n0 : after);
        rcd.terms_gained = rcd.terms_after - std::min(rcd.terms_after, rcd.terms_before);
        if (op >= 0) {
          if (P.log) {
            const u64* w = &lg[(size_t)op * pq::LOG_WORDS];
            rcd.declined = w[pq::LOG_HELD];
            rcd.emitted = w[pq::LOG_EMITTED];
            rcd.exchange_hits = w[pq::LOG_HITS];
            std::memcpy(&rcd.discarded_coeff_l1, &w[pq::LOG_L1], 8);
            std::memcpy(&rcd.discarded_coeff_max, &w[pq::LOG_MAX], 8);
          }
          // the op's device time; a fused op's time goes to its first rotation
          rcd.elapsed_ms = op > 0 && stamps[op] > stamps[op - 1] ? (double)(stamps[op] - stamps[op - 1]) * 1e-6 : 0.0;
        }
      }
  }
  for (size_t i = 0; i < no; ++i) {
    if (pq::is_class(P.ops[i].kind)) ++res->class_ops;
    const u64 n_in = i ? hist[i - 1] : P.n0;
    const double op_ms = i && stamps[i] > stamps[i - 1] ? (double)(stamps[i] - stamps[i - 1]) * 1e-6 : 0.0;
    switch (pq::is_class(P.ops[i].kind) ? (u32)pq::OP_GATE : P.ops[i].kind) {
      case pq::OP_GATE:
      case pq::OP_GATE2:
      case pq::OP_GATE3:
      case pq::OP_GATE4:
      case pq::OP_GATE_TAIL:
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
        res->sum_kept += P.ops[i].kind == pq::OP_NOISE_COMPACT ? hist[i] : 0;
    }
  }
  res->sweep_ms = P.sweep_ms;
  res->sweep_launches = P.sweep_launches;
  res->n_final = P.n_live;
  res->peak_terms = P.peak;
  res->sparse_key_bytes = P.n_live * P.W * 8 + S.tcap * 8;
  res->n_layers_run = in.n_layers;
  res->n_gates_run = in.n_gates;
  return PQ_OK;
}

int run_one(pq_engine* E, const Inputs& in, int W) {
  if (int rc = E->ensure_slots(1)) return rc;
  Slot& S = E->slots[0];
  Plan P;
  if (int rc = prepare(E, P, in, W)) return rc;
  if (int rc = setup_slot(E, S, P)) return rc;
  const int grid = with_words(W, [&](auto w) {
    constexpr int WW = decltype(w)::value;
    return P.alg == 0 ? pq::sweep_grid<WW, 0>((int)in.cfg->blocks_per_sm)
                      : pq::sweep_grid<WW, 1>((int)in.cfg->blocks_per_sm);
  });
  bool began = false;
  auto need_n = [&](u64* n) -> int {
    if (int rc = execute_single(E, S, P, grid, &began)) return rc;
    *n = P.n_live;
    return PQ_OK;
  };
  if (int rc = build_ops(P, need_n)) return rc;
  fuse_classes(P);
  fuse_groups(P);
  if (int rc = execute_single(E, S, P, grid, &began)) return rc;
  if (!began) cudaEventRecord(E->ev_begin, E->stream);
  std::vector<pq::ExpectPartial> parts;
  if (int rc = finalize(E, S, P, &parts)) return rc;
  cudaEventRecord(E->ev_end, E->stream);
  if (cudaError_t e = cudaStreamSynchronize(E->stream)) return E->cuda_fail(e, "finalize");
  if (int rc = finish(E, S, P, parts)) return rc;
  float ms = 0;
  cudaEventElapsedTime(&ms, E->ev_begin, E->ev_end);
  in.res->device_ms = ms;
  return PQ_OK;
}

// Expectation value and dE/d(angle) of every gate with the truncation
// decisions of the forward run held fixed.  The forward run records each op
// (SweepArgs::rec_idx: sin-branch partners, pre-op coefficients, reclaim maps
// and key snapshots) into a pool of record_bytes (0: what the last such
// gradient needed plus a quarter, at first 40% of the free device memory, at
// most 48 GB; the engine keeps the pool) and keeps the live terms at the start of every
// segment of ckpt_layers layers.  If every op fit, one reverse sweep
// (adjoint_kernel) carries dE/dc from the final rows back to the observable.
// If the pool ran out, the reverse pass goes segment by segment, last first:
// restore the segment's start, run it again recording from the start of the
// pool, sweep it in reverse.  Records take 12 bytes per row entering each op
// (plus 8W per row entering a reclaim).
int run_adjoint(pq_engine* E, const Inputs& in, int W, u32 ckpt_layers, u64 record_bytes, double* grad_out) {
  if (!in.diag) return E->fail(PQ_ERR_INVALID, "the gradient needs an initial state");
  if (int rc = E->ensure_slots(1)) return rc;
  Slot& S = E->slots[0];
  Plan P;
  if (int rc = prepare(E, P, in, W)) return rc;
  if (P.host_ops)
    return E->fail(PQ_ERR_UNSUPPORTED, "the gradient does not run truncator plugins or key-reading noise");
  if (int rc = setup_slot(E, S, P)) return rc;
  const int ALG = P.alg;
  const int grid = with_words(W, [&](auto w) {
    constexpr int WW = decltype(w)::value;
    return ALG == 0 ? pq::sweep_grid<WW, 0>((int)in.cfg->blocks_per_sm)
                    : pq::sweep_grid<WW, 1>((int)in.cfg->blocks_per_sm);
  });
  const int agrid = with_words(W, [&](auto w) {
    constexpr int WW = decltype(w)::value;
    return ALG == 0 ? pq::adjoint_grid<WW, 0>() : pq::adjoint_grid<WW, 1>();
  });
  auto no_sync = [&](u64*) -> int {
    return E->fail(PQ_ERR_UNSUPPORTED,
                   "the gradient cannot decide Clifford deferral under a TermBudget floor with a weight cut");
  };
  if (int rc = build_ops(P, no_sync)) return rc;
  const size_t n_ops = P.ops.size();
  const size_t per = ckpt_layers ? ckpt_layers : std::max<size_t>(in.n_layers, 1);
  std::vector<size_t> seg;
  for (size_t l = 0; l < in.n_layers; l += per) seg.push_back(P.layer_op[l]);
  seg.push_back(n_ops);
  const size_t n_seg = seg.size() - 1;
  cudaError_t e;

  // The record pool, split between the per-row records (12 B an element) and
  // reclaim key snapshots: record_bytes, else the size the last default-sized
  // gradient needed (plus a quarter), else 40% of the free device memory (at
  // most 48 GB).  The engine keeps it for the next gradient.
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const size_t ceiling = std::min<size_t>((free_b + E->g_pool.bytes) / 5 * 2, (size_t)48 << 30);
  Recording rec;
  auto setup_pool = [&](size_t budget) -> cudaError_t {
    rec.cap = std::max<u64>(budget / 100 * 85 / 12, 1);
    rec.key_cap = std::max<u64>(budget / 100 * 15 / (8 * (size_t)W), 1);
    const size_t o_coef = align256(4 * rec.cap), o_keys = o_coef + align256(8 * rec.cap),
                 o_off = o_keys + align256(8 * (size_t)W * rec.key_cap), o_koff = o_off + align256(8 * n_ops),
                 pool_end = o_koff + align256(8 * n_ops);
    if (E->g_pool.bytes < pool_end) E->g_pool.release();  // before the new one, so both never coexist
    if (cudaError_t ee = E->g_pool.ensure(pool_end)) return ee;
    rec.idx = E->g_pool.at<u32>(0);
    rec.coef = E->g_pool.at<double>(o_coef);
    rec.keys = E->g_pool.at<u64>(o_keys);
    rec.off = E->g_pool.at<u64>(o_off);
    rec.key_off = E->g_pool.at<u64>(o_koff);
    return cudaSuccess;
  };
  size_t budget = record_bytes ? (size_t)record_bytes : (E->g_need ? std::min(E->g_need / 4 * 5, ceiling) : ceiling);
  if ((e = setup_pool(budget)) != cudaSuccess) return E->cuda_fail(e, "gradient record pool");

  // Forward, keeping each segment's starting terms and recording every op
  // while the pool lasts.
  std::vector<u64*> ck_keys(n_seg, nullptr);
  std::vector<double*> ck_coeffs(n_seg, nullptr);
  std::vector<u64> ck_n(n_seg, 0);
  if (E->g_ck.size() < n_seg) E->g_ck.resize(n_seg);
  bool began = false;
  P.rec_next = P.rec_key_next = 0;
  P.rec_full = 0;
  for (size_t s = 0; s < n_seg; ++s) {
    ck_n[s] = P.n_live;
    const size_t o_c = align256(8 * (size_t)W * ck_n[s]);
    if ((e = E->g_ck[s].ensure(o_c + 8 * ck_n[s])) != cudaSuccess) return E->cuda_fail(e, "checkpoint");
    ck_keys[s] = E->g_ck[s].at<u64>(0);
    ck_coeffs[s] = E->g_ck[s].at<double>(o_c);
    cudaMemcpyAsync(ck_keys[s], S.keys[S.cur], ck_n[s] * W * 8, cudaMemcpyDeviceToDevice, E->stream);
    cudaMemcpyAsync(ck_coeffs[s], S.coeffs[S.cur], ck_n[s] * 8, cudaMemcpyDeviceToDevice, E->stream);
    if (int rc = execute_single(E, S, P, grid, &began, seg[s + 1], &rec)) return rc;
  }
  const bool recorded_all = !P.rec_full;
  if (!began) cudaEventRecord(E->ev_begin, E->stream);
  std::vector<pq::ExpectPartial> parts;
  if (int rc = finalize(E, S, P, &parts)) return rc;
  if ((e = cudaStreamSynchronize(E->stream)) != cudaSuccess) return E->cuda_fail(e, "expectation");
  if (int rc = finish(E, S, P, parts)) return rc;
  const u64 n_fin = P.n_live;

  // Rows entering each op, gate -> op map, adjoint buffers.
  std::vector<u64> hist(n_ops), n_in(n_ops), koff(n_ops, 0);
  if (n_ops) cudaMemcpy(hist.data(), S.hist, n_ops * 8, cudaMemcpyDeviceToHost);
  for (size_t k = 0; k < n_ops; ++k) n_in[k] = k ? hist[k - 1] : P.n0;
  if (!record_bytes) {  // the pool that records every op of this run
    u64 rows = 0, keys = 0;
    for (size_t k = 0; k < n_ops; ++k) {
      if (P.ops[k].kind == pq::OP_NOISE_SCALE) continue;
      rows += n_in[k];
      if (P.ops[k].kind == pq::OP_NOISE_COMPACT) keys += n_in[k];
    }
    E->g_need = std::max<size_t>(rows * 12 / 85 * 100 + 100, keys * 8 * (size_t)W / 15 * 100 + 100);
    // A default pool sized for an earlier, smaller problem: grow it to this
    // run's need before the segments are re-run to record them.
    const size_t want = std::min(E->g_need / 4 * 5, ceiling);
    if (!recorded_all && want > budget) {
      budget = want;
      if ((e = setup_pool(budget)) != cudaSuccess) return E->cuda_fail(e, "gradient record pool");
    }
  }
  std::vector<long long> gate_ops(in.n_gates);
  for (size_t g = 0; g < in.n_gates; ++g) gate_ops[g] = P.gate_own[g] ? P.gate_op[g] : -1;
  double* lam[2] = {nullptr, nullptr};
  double* grad_part = nullptr;
  double* d_grad = nullptr;
  u64* d_n_in = nullptr;
  long long* d_gate_ops = nullptr;
  const u64** d_ksrc = nullptr;
  if ((e = E->g_lam.ensure(align256(8 * S.cap) * 2)) != cudaSuccess) return E->cuda_fail(e, "adjoint vectors");
  lam[0] = E->g_lam.at<double>(0);
  lam[1] = E->g_lam.at<double>(align256(8 * S.cap));
  {
    const size_t o_grad = align256(8 * n_ops * (size_t)agrid), o_nin = o_grad + align256(8 * in.n_gates),
                 o_gops = o_nin + align256(8 * n_ops), o_ksrc = o_gops + align256(8 * in.n_gates),
                 end = o_ksrc + align256(8 * n_ops);
    if ((e = E->g_ops.ensure(end)) != cudaSuccess) return E->cuda_fail(e, "adjoint buffers");
    grad_part = E->g_ops.at<double>(0);
    d_grad = E->g_ops.at<double>(o_grad);
    d_n_in = E->g_ops.at<u64>(o_nin);
    d_gate_ops = E->g_ops.at<long long>(o_gops);
    d_ksrc = E->g_ops.at<const u64*>(o_ksrc);
  }
  if (n_ops) {
    cudaMemcpyAsync(d_n_in, n_in.data(), n_ops * 8, cudaMemcpyHostToDevice, E->stream);
    cudaMemsetAsync(grad_part, 0, n_ops * (size_t)agrid * 8, E->stream);
  }
  if (in.n_gates)
    cudaMemcpyAsync(d_gate_ops, gate_ops.data(), in.n_gates * 8, cudaMemcpyHostToDevice, E->stream);

  // Seed: dE/dc of the final rows.
  const pq::ExpectArgs xa = expect_args(S, P);
  ++E->launches;
  e = with_words(W, [&](auto w) {
    constexpr int WW = decltype(w)::value;
    return ALG == 0 ? pq::launch_adjoint_seed<WW, 0>(xa, S.keys[S.cur], n_fin, lam[0], E->stream)
                    : pq::launch_adjoint_seed<WW, 1>(xa, S.keys[S.cur], n_fin, lam[0], E->stream);
  });
  if (e != cudaSuccess) return E->cuda_fail(e, "adjoint seed");
  int lam_cur = 0;

  // The reverse sweep over ops [b, e): keys of each op's input rows are the
  // snapshot of the next reclaim (rows only grow until then), else the buffer
  // the rows ended in.
  auto reverse = [&](size_t b, size_t end_op, const u64* last_keys) -> int {
    if (b == end_op) return PQ_OK;
    cudaMemcpyAsync(koff.data() + b, rec.key_off + b, (end_op - b) * 8, cudaMemcpyDeviceToHost, E->stream);
    cudaError_t ee;
    if ((ee = cudaStreamSynchronize(E->stream)) != cudaSuccess) return E->cuda_fail(ee, "record offsets");
    std::vector<const u64*> ksrc(end_op - b);
    const u64* next = last_keys;
    for (size_t k = end_op; k-- > b;) {
      if (P.ops[k].kind == pq::OP_NOISE_COMPACT) next = rec.keys + koff[k] * W;
      ksrc[k - b] = next;
    }
    cudaMemcpyAsync(d_ksrc + b, ksrc.data(), ksrc.size() * sizeof(u64*), cudaMemcpyHostToDevice, E->stream);
    E->h_states[0] = pq::SweepState{};
    E->init_waits(E->h_states[0]);
    cudaMemcpyAsync(E->d_states, E->h_states, sizeof(pq::SweepState), cudaMemcpyHostToDevice, E->stream);
    pq::AdjointArgs aa{};
    aa.ops = S.d_ops;
    aa.gates = S.d_gates;
    aa.tables = S.d_tables;
    aa.table_len = (u32)P.tlen;
    aa.n_units = P.n_units;
    aa.op_begin = (u32)b;
    aa.op_end = (u32)end_op;
    aa.cur0 = (u32)lam_cur;
    aa.n_in = d_n_in;
    aa.rec_idx = rec.idx;
    aa.rec_coef = rec.coef;
    aa.rec_off = rec.off;
    aa.key_src = d_ksrc;
    aa.lam[0] = lam[0];
    aa.lam[1] = lam[1];
    aa.grad_part = grad_part;
    aa.st = E->d_states;
    ++E->launches;
    ee = with_words(W, [&](auto w) {
      constexpr int WW = decltype(w)::value;
      return ALG == 0 ? pq::launch_adjoint<WW, 0>(aa, agrid, E->stream) : pq::launch_adjoint<WW, 1>(aa, agrid, E->stream);
    });
    if (ee != cudaSuccess) return E->cuda_fail(ee, "adjoint launch");
    cudaMemcpyAsync(E->h_states, E->d_states, sizeof(pq::SweepState), cudaMemcpyDeviceToHost, E->stream);
    if ((ee = cudaStreamSynchronize(E->stream)) != cudaSuccess) return E->cuda_fail(ee, "adjoint");
    if (E->h_states[0].error & pq::ERR_BARRIER_TIMEOUT)
      return E->fail(PQ_ERR_DEVICE_TIMEOUT, "a grid barrier wait expired on the device");
    if (E->h_states[0].error)
      return E->fail(PQ_ERR_CUDA, "device reported error bits " + std::to_string(E->h_states[0].error));
    lam_cur = (int)E->h_states[0].cur;
    return PQ_OK;
  };

  if (recorded_all) {
    // Every op was recorded in the forward pass: one reverse sweep, no replay.
    if (int rc = reverse(0, n_ops, S.keys[S.cur])) return rc;
  } else {
    // The pool ran out: last segment first, restore its start, run it again
    // recording from the start of the pool, then sweep it in reverse.
    for (size_t sg = n_seg; sg-- > 0;) {
      if (seg[sg] == seg[sg + 1]) continue;
      if (ck_n[sg]) {
        cudaMemcpyAsync(S.keys[0], ck_keys[sg], ck_n[sg] * W * 8, cudaMemcpyDeviceToDevice, E->stream);
        cudaMemcpyAsync(S.coeffs[0], ck_coeffs[sg], ck_n[sg] * 8, cudaMemcpyDeviceToDevice, E->stream);
      }
      S.cur = 0;
      if (int rc = E->rebuild_table(S, ck_n[sg])) return rc;
      P.done = seg[sg];
      P.n_live = ck_n[sg];
      P.rec_next = P.rec_key_next = 0;
      P.rec_full = 0;
      if (int rc = execute_single(E, S, P, grid, &began, seg[sg + 1], &rec)) return rc;
      if (P.rec_full)
        return E->fail(PQ_ERR_OOM, "one segment's gradient records exceed the device memory set aside for them; "
                                   "use fewer checkpoint layers");
      if (int rc = reverse(seg[sg], seg[sg + 1], S.keys[S.cur])) return rc;
    }
  }
  ++E->launches;
  if ((e = pq::launch_grad_reduce(grad_part, agrid, d_gate_ops, in.n_gates, d_grad, E->stream)) != cudaSuccess)
    return E->cuda_fail(e, "gradient reduction");
  if (in.n_gates) cudaMemcpyAsync(grad_out, d_grad, in.n_gates * 8, cudaMemcpyDeviceToHost, E->stream);
  cudaEventRecord(E->ev_end, E->stream);
  if ((e = cudaStreamSynchronize(E->stream)) != cudaSuccess) return E->cuda_fail(e, "gradient");
  float ms = 0;
  cudaEventElapsedTime(&ms, E->ev_begin, E->ev_end);
  in.res->device_ms = ms;
  // A default-sized pool far above what this run needed is given back; the
  // next gradient allocates the measured size.
  if (!record_bytes && E->g_pool.bytes / 2 > E->g_need / 4 * 5 + 32 * n_ops) E->g_pool.release();
  return PQ_OK;
}

// Splits `blocks` among the instances in `todo`: one each, the rest equally
// (split 0) or in proportion to remaining ops x (live terms + units), the work
// still ahead if the live count stayed where it is (split 1).
std::vector<u32> share_blocks(const std::vector<Plan>& plans, const std::vector<size_t>& todo, size_t blocks,
                              u32 split) {
  std::vector<double> wgt(todo.size(), 1.0);
  if (split == 1)
    for (size_t k = 0; k < todo.size(); ++k) {
      const Plan& P = plans[todo[k]];
      wgt[k] = (double)(P.ops.size() - P.done) * ((double)P.n_live + (double)P.n_units);
    }
  double wsum = 0;
  for (double w : wgt) wsum += w;
  std::vector<u32> cnt(todo.size(), 1);
  const size_t spare = blocks - todo.size();
  size_t given = 0;
  for (size_t k = 0; k < todo.size() && wsum > 0; ++k) {
    const u32 extra = (u32)std::floor((double)spare * wgt[k] / wsum);
    cnt[k] += extra;
    given += extra;
  }
  for (size_t k = 0; given < spare; k = (k + 1) % todo.size(), ++given) ++cnt[k];
  return cnt;
}

// A batch in cooperative launches of batch_sweep_kernel: every unfinished
// instance gets a contiguous slice of the grid (at least one block) and runs
// its own op sequence with its own barrier.  When rebalance_pct of the grid
// has been left by instances that finished (or stopped for capacity), the
// rest stop at their next op boundary and the next launch re-splits the whole
// grid among the instances still running; instances that halted for capacity
// are grown first.
int run_batch(pq_engine* E, const std::vector<Inputs>& ins, int WM, const pq_batch_tuning& tune) {
  const size_t n = ins.size();
  const int alg = (int)ins[0].cfg->basis_kind;
  if (int rc = E->ensure_slots(n)) return rc;
  std::vector<Plan> plans(n);
  auto no_sync = [&](u64*) -> int {
    return E->fail(PQ_ERR_UNSUPPORTED,
                   "a batch cannot decide Clifford deferral under a TermBudget floor with a weight cut; run that "
                   "instance with pq_run");
  };
  for (size_t i = 0; i < n; ++i) {
    const int W = std::max(ins[i].in_words, WM > 1 ? WM / 2 : 1);
    if (int rc = prepare(E, plans[i], ins[i], W)) return rc;
    if (plans[i].host_ops)
      return E->fail(PQ_ERR_UNSUPPORTED, "a batch does not run truncator plugins or key-reading noise; use pq_run");
    if (tune.fuse_max) plans[i].fuse_max = tune.fuse_max;
    if (tune.tile_items) plans[i].tile_items = tune.tile_items;
    if (tune.bucket_slots) plans[i].bucket_slots = tune.bucket_slots;
    if (int rc = setup_slot(E, E->slots[i], plans[i])) return rc;
    if (int rc = build_ops(plans[i], no_sync)) return rc;
    fuse_classes(plans[i]);
    fuse_groups(plans[i]);
    upload_ops(E, E->slots[i], plans[i]);
  }
  const int grid_max = with_words(WM, [&](auto w) {
    constexpr int WW = decltype(w)::value;
    return alg == 0 ? pq::batch_grid<WW, 0>((int)tune.blocks_per_sm) : pq::batch_grid<WW, 1>((int)tune.blocks_per_sm);
  });
  if (int rc = E->ensure_batch_arrays(n, (size_t)grid_max)) return rc;
  cudaError_t e;
  bool began = false;
  double sweep_ms = 0;
  std::vector<size_t> todo;
  for (;;) {
    todo.clear();
    for (size_t i = 0; i < n && todo.size() < (size_t)grid_max; ++i)
      if (plans[i].done < plans[i].ops.size()) todo.push_back(i);
    if (todo.empty()) break;
    const std::vector<u32> cnt = share_blocks(plans, todo, (size_t)grid_max, tune.split);
    // One instance left: nothing to re-split.
    const bool rebalance = tune.rebalance_pct > 0 && todo.size() > 1;
    const u32 yield_at = std::max<u32>(1, (u32)((u64)grid_max * std::min<u32>(tune.rebalance_pct, 100) / 100));
    u32 off = 0;
    for (size_t k = 0; k < todo.size(); ++k) {
      Slot& S = E->slots[todo[k]];
      Plan& P = plans[todo[k]];
      if (P.has_class)
        if (int rc = E->ensure_class(S)) return rc;
      E->h_states[k] = fresh_state(E, P);
      cudaMemsetAsync(S.tickets + P.done, 0, (P.ops.size() - P.done) * 4, E->stream);
      E->h_args[k] = sweep_args(S, P, E->d_states + k, off, cnt[k]);
      E->limit_args(E->h_args[k]);
      E->h_args[k].idle_blocks = rebalance ? E->d_idle : nullptr;
      E->h_args[k].yield_at = yield_at;
      for (u32 b = 0; b < cnt[k]; ++b) E->h_block_inst[off + b] = (u32)k;
      off += cnt[k];
    }
    cudaMemcpyAsync(E->d_states, E->h_states, todo.size() * sizeof(pq::SweepState), cudaMemcpyHostToDevice,
                    E->stream);
    cudaMemcpyAsync(E->d_args, E->h_args, todo.size() * sizeof(pq::SweepArgs), cudaMemcpyHostToDevice, E->stream);
    cudaMemcpyAsync(E->d_block_inst, E->h_block_inst, off * 4, cudaMemcpyHostToDevice, E->stream);
    cudaMemsetAsync(E->d_idle, 0, sizeof(u32), E->stream);
    if (!began) {
      cudaEventRecord(E->ev_begin, E->stream);
      began = true;
    }
    cudaEventRecord(E->ev_l0, E->stream);
    e = with_words(WM, [&](auto w) {
      constexpr int WW = decltype(w)::value;
      return alg == 0 ? pq::launch_batch_sweep<WW, 0>(E->d_args, E->d_block_inst, (int)off, E->stream)
                      : pq::launch_batch_sweep<WW, 1>(E->d_args, E->d_block_inst, (int)off, E->stream);
    });
    if (e != cudaSuccess) return E->cuda_fail(e, "batch sweep launch");
    cudaEventRecord(E->ev_l1, E->stream);
    ++E->launches;
    cudaMemcpyAsync(E->h_states, E->d_states, todo.size() * sizeof(pq::SweepState), cudaMemcpyDeviceToHost,
                    E->stream);
    if ((e = cudaStreamSynchronize(E->stream)) != cudaSuccess) return E->cuda_fail(e, "batch sweep");
    float ms = 0;
    cudaEventElapsedTime(&ms, E->ev_l0, E->ev_l1);
    sweep_ms += ms;
    for (size_t k = 0; k < todo.size(); ++k)
      if (int rc = absorb_state(E, E->slots[todo[k]], plans[todo[k]], E->h_states[k])) return rc;
  }
  if (!began) cudaEventRecord(E->ev_begin, E->stream);
  std::vector<std::vector<pq::ExpectPartial>> parts(n);
  for (size_t i = 0; i < n; ++i)
    if (int rc = finalize(E, E->slots[i], plans[i], &parts[i])) return rc;
  cudaEventRecord(E->ev_end, E->stream);
  if ((e = cudaStreamSynchronize(E->stream)) != cudaSuccess) return E->cuda_fail(e, "finalize");
  float ms = 0;
  cudaEventElapsedTime(&ms, E->ev_begin, E->ev_end);
  for (size_t i = 0; i < n; ++i) {
    if (int rc = finish(E, E->slots[i], plans[i], parts[i])) return rc;
    ins[i].res->device_ms = ms;  // the batch's device time
    ins[i].res->sweep_ms = sweep_ms;
  }
  return PQ_OK;
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
  if (dmalloc(&E->d_err, sizeof(u32)) != cudaSuccess) return PQ_ERR_OOM;
  if (dmalloc(&E->d_idle, sizeof(u32)) != cudaSuccess) return PQ_ERR_OOM;
  cudaMemset(E->d_err, 0, sizeof(u32));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  E->expect_grid = 4 * sms;
  for (cudaEvent_t* ev : {&E->ev_begin, &E->ev_end, &E->ev_l0, &E->ev_l1}) cudaEventCreate(ev);
  if (E->ensure_slots(1) != PQ_OK) return PQ_ERR_OOM;
  *out = E.release();
  return PQ_OK;
}

void pq_engine_destroy(pq_engine* E) {
  BudgetScope scope(E ? &E->budget : nullptr);
  delete E;
}

int pq_engine_set_limits(pq_engine* E, const pq_engine_limits* lim) {
  if (!E) return PQ_ERR_INVALID;
  E->lim = lim ? *lim : pq_engine_limits{};
  E->budget.limit = (size_t)E->lim.max_device_bytes;
  return PQ_OK;
}

uint64_t pq_engine_device_bytes(const pq_engine* E) { return E ? (uint64_t)E->budget.used : 0; }
const char* pq_engine_last_error(const pq_engine* E) { return E ? E->err.c_str() : "null engine"; }

}  // extern "C"

namespace {

// Argument checks shared by pq_run and pq_run_batch; sets the key width.
int check_inputs(pq_engine* E, const pq_run_config* cfg, size_t ng, const uint32_t* lo, size_t nl, int* W_out) {
  if (cfg->basis_kind > 1) return E->fail(PQ_ERR_INVALID, "basis_kind must be 0 (Pauli) or 1 (Majorana)");
  const uint32_t W = pq_words_for_units(cfg->n_units);
  if (!W)
    return E->fail(PQ_ERR_INVALID, "propaq: " + std::to_string(cfg->n_units) +
                                       " units exceeds the engine's maximum of 2048");
  if (cfg->fuse_max > pq::GROUP_MAX) return E->fail(PQ_ERR_INVALID, "fuse_max must be 0..2");
  if (cfg->tile_items > 4) return E->fail(PQ_ERR_INVALID, "tile_items must be 0..4");
  if (cfg->bucket_slots != 0 && cfg->bucket_slots != 2 && cfg->bucket_slots != 4 && cfg->bucket_slots != 8)
    return E->fail(PQ_ERR_INVALID, "bucket_slots must be 0, 2, 4 or 8");
  if (nl && (!lo || lo[0] != 0 || lo[nl] != ng)) return E->fail(PQ_ERR_INVALID, "layer offsets do not cover the gates");
  if (!nl && ng) return E->fail(PQ_ERR_INVALID, "layer offsets do not cover the gates");
  for (size_t l = 0; l < nl; ++l)
    if (lo[l + 1] < lo[l]) return E->fail(PQ_ERR_INVALID, "layer offsets must be non-decreasing");
  *W_out = (int)W;
  return PQ_OK;
}

// uint64_t and the kernels' unsigned long long are both 64-bit words.
inline const u64* K(const uint64_t* p) { return reinterpret_cast<const u64*>(p); }

}  // namespace

extern "C" {

int pq_run(pq_engine* E, const pq_run_config* cfg, const uint64_t* ow, const double* oc, size_t no,
           const uint64_t* gw, const double* ga, size_t ng, const uint32_t* lo, size_t nl, const uint64_t* d,
           size_t nd, uint64_t* nt, pq_result* r) {
  BudgetScope scope(E ? &E->budget : nullptr);
  if (!E || !cfg || !r) return PQ_ERR_INVALID;
  std::memset(r, 0, sizeof(*r));
  E->err.clear();
  int W = 0;
  if (int rc = check_inputs(E, cfg, ng, lo, nl, &W)) return rc;
  if (cudaSetDevice(E->device) != cudaSuccess) return E->fail(PQ_ERR_CUDA, "cudaSetDevice failed");
  const u64 l0 = E->launches;
  const Inputs in{cfg, K(ow), oc, no, K(gw), ga, ng, lo, nl, K(d), nd, reinterpret_cast<u64*>(nt), r, W};
  const int rc = run_one(E, in, W);
  r->gpu_launches = E->launches - l0;
  return rc;
}

int pq_run_batch(pq_engine* E, const pq_instance* insts, size_t n, const pq_batch_tuning* tuning) {
  BudgetScope scope(E ? &E->budget : nullptr);
  if (!E || !insts || !n) return PQ_ERR_INVALID;
  E->err.clear();
  const pq_batch_tuning tune = tuning ? *tuning : pq_batch_tuning{0, 1, 25, 0, 0, 0};
  if (tune.split > 1) return E->fail(PQ_ERR_INVALID, "split must be 0 (equal) or 1 (by remaining work)");
  if (tune.fuse_max > pq::GROUP_MAX) return E->fail(PQ_ERR_INVALID, "fuse_max must be 0..2");
  if (tune.tile_items > 4) return E->fail(PQ_ERR_INVALID, "tile_items must be 0..4");
  if (tune.bucket_slots != 0 && tune.bucket_slots != 2 && tune.bucket_slots != 4 && tune.bucket_slots != 8)
    return E->fail(PQ_ERR_INVALID, "bucket_slots must be 0, 2, 4 or 8");
  if (tune.rebalance_pct > 100) return E->fail(PQ_ERR_INVALID, "rebalance_pct must be 0..100");
  const uint32_t basis = insts[0].cfg.basis_kind;
  int WM = 1;
  std::vector<Inputs> ins(n);
  for (size_t i = 0; i < n; ++i) {
    const pq_instance& x = insts[i];
    if (!x.result) return E->fail(PQ_ERR_INVALID, "instance " + std::to_string(i) + " has no result");
    std::memset(x.result, 0, sizeof(pq_result));
    if (x.cfg.basis_kind != basis) return E->fail(PQ_ERR_INVALID, "a batch mixes Pauli and Majorana instances");
    int W = 0;
    if (int rc = check_inputs(E, &x.cfg, x.n_gates, x.layer_offsets, x.n_layers, &W)) return rc;
    WM = std::max(WM, W);
    ins[i] = Inputs{&x.cfg,          K(x.obs_words),  x.obs_coeffs,  x.n_obs,
                    K(x.gate_words), x.gate_angles,   x.n_gates,     x.layer_offsets,
                    x.n_layers,      K(x.diag_state), x.diag_words,  reinterpret_cast<u64*>(x.n_terms_out),
                    x.result,        W};
  }
  if (cudaSetDevice(E->device) != cudaSuccess) return E->fail(PQ_ERR_CUDA, "cudaSetDevice failed");
  const u64 l0 = E->launches;
  const int rc = run_batch(E, ins, WM, tune);
  for (size_t i = 0; i < n; ++i) insts[i].result->gpu_launches = E->launches - l0;
  return rc;
}

int pq_run_adjoint(pq_engine* E, const pq_run_config* cfg, const uint64_t* ow, const double* oc, size_t no,
                   const uint64_t* gw, const double* ga, size_t ng, const uint32_t* lo, size_t nl, const uint64_t* d,
                   size_t nd, uint32_t checkpoint_layers, uint64_t record_bytes, double* grad, uint64_t* nt,
                   pq_result* r) {
  BudgetScope scope(E ? &E->budget : nullptr);
  if (!E || !cfg || !r || (ng && !grad)) return PQ_ERR_INVALID;
  std::memset(r, 0, sizeof(*r));
  E->err.clear();
  int W = 0;
  if (int rc = check_inputs(E, cfg, ng, lo, nl, &W)) return rc;
  if (cudaSetDevice(E->device) != cudaSuccess) return E->fail(PQ_ERR_CUDA, "cudaSetDevice failed");
  const u64 l0 = E->launches;
  const Inputs in{cfg, K(ow), oc, no, K(gw), ga, ng, lo, nl, K(d), nd, reinterpret_cast<u64*>(nt), r, W};
  const int rc = run_adjoint(E, in, W, checkpoint_layers, record_bytes, grad);
  r->gpu_launches = E->launches - l0;
  return rc;
}

size_t pq_result_terms_at(pq_engine* E, size_t index, uint64_t* keys, double* coeffs, size_t cap) {
  if (!E || index >= E->slots.size()) return 0;
  const Slot& S = E->slots[index];
  const size_t n = S.out_coeffs.size();
  const size_t m = std::min(n, cap);
  if (m) {
    std::memcpy(keys, S.out_keys.data(), m * S.out_words * 8);
    std::memcpy(coeffs, S.out_coeffs.data(), m * 8);
  }
  return n;
}

size_t pq_result_terms(pq_engine* E, uint64_t* keys, double* coeffs, size_t cap) {
  return pq_result_terms_at(E, 0, keys, coeffs, cap);
}

size_t pq_result_gates(pq_engine* E, pq_gate_record* out, size_t cap) {
  if (!E || E->slots.empty()) return 0;
  const std::vector<pq_gate_record>& g = E->slots[0].gate_log;
  const size_t m = std::min(g.size(), cap);
  if (m && out) std::memcpy(out, g.data(), m * sizeof(pq_gate_record));
  return g.size();
}

int pq_plugin_load_noise(const char* path, const char* cfg, pq_plugin** out, char* err, size_t n) {
  return load_plugin(true, path, cfg, out, err, n);
}
int pq_plugin_load_truncator(const char* path, const char* cfg, pq_plugin** out, char* err, size_t n) {
  return load_plugin(false, path, cfg, out, err, n);
}
void pq_plugin_free(pq_plugin* p) { delete reinterpret_cast<Plugin*>(p); }

int pq_plugin_from_callback(pq_noise_factor_fn fn, void* ctx, uint32_t depends, pq_plugin** out) {
  if (!fn || !out) return PQ_ERR_INVALID;
  if (depends & ~3u) return PQ_ERR_PLUGIN;
  auto* p = new Plugin;
  p->noise = true;
  p->ctx = ctx;
  p->depends = depends;
  p->fn = reinterpret_cast<void*>(fn);
  *out = reinterpret_cast<pq_plugin*>(p);
  return PQ_OK;
}
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
