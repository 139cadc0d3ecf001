// pq_kernels.cu -- the hot path of the B200 propagation engine.
//
// One gate is ONE persistent kernel (gate_kernel).  It replaces the
// reference's scan -> route -> absorb -> claim -> rescue rounds
// (crates/core/src/engine/partitioned_termsum.rs:276-450,
//  crates/core/src/engine/termsum.rs:561-800) with a single pass:
//
//   * each row is tested for anticommutation by popcount parity;
//   * an anticommuting row looks its child K = G.S up in the open-addressing
//     hash table (pre-gate rows only).  K -> G.K is an involution, so a row
//     has at most one partner; the lower row of a pair owns both
//     coefficients and applies the pair rule to both, reading the pre-gate
//     values, so no coefficient is ever written by two threads;
//   * a lone row whose branch survives the emit cutoff creates its child;
//     children are appended in row order through a warp-ballot / block scan
//     and a decoupled look-back across tiles, and inserted into the table by
//     atomicCAS on the packed (fingerprint, row) slot.
//
// Rows are never removed by a gate; a noisy layer's reclaim (noise_kernel)
// damps, filters and compacts them in row order into the ping-pong buffers
// and re-inserts the survivors into a cleared table.
//
// Every kernel uses the same persistent-grid protocol: it reads the live
// count of the current parity from the device control block at entry, takes
// tiles from an atomic ticket, and the last block to leave publishes the new
// count and resets the counters.  All spin-waits are bounded and raise an
// error bit instead of hanging.
#include <cuda_runtime.h>

#include <cstdio>

#include "pq_kernels.cuh"

namespace pq {

namespace {

constexpr int BLOCK = 256;
constexpr int NWARPS = BLOCK / 32;
constexpr int ITEMS = 4;  // rows per thread per tile; ITEMS * NWARPS == 32
constexpr int TILE = BLOCK * ITEMS;
static_assert(ITEMS * NWARPS == 32, "tile scan uses one warp");

constexpr u32 ST_AGG = 1u, ST_INC = 2u;
constexpr unsigned FULL = 0xffffffffu;
constexpr long LOOKBACK_SPIN_LIMIT = 1L << 22;  // ~0.3 s with the backoff below

enum : int { S_EMIT = 0, S_HELD = 1, S_DROP = 2 };

__device__ __forceinline__ u64 pack_status(u32 epoch, u32 flag, u32 value) {
  return ((u64)(epoch & 0x3fffffffu) << 34) | ((u64)flag << 32) | value;
}

__device__ __forceinline__ u64 ld_volatile(const u64* p) { return *(const volatile u64*)p; }
__device__ __forceinline__ void st_volatile(u64* p, u64 v) { *(volatile u64*)p = v; }

// Decoupled look-back (called by all lanes of warp 0): publishes this tile's
// aggregate, walks predecessors 32 at a time, returns the exclusive prefix.
__device__ u32 lookback(u64* status, u32 tile, u32 agg, u32 epoch, Ctl* ctl) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) st_volatile(&status[0], pack_status(epoch, ST_INC, agg));
    return 0;
  }
  if (lane == 0) st_volatile(&status[tile], pack_status(epoch, ST_AGG, agg));
  u32 excl = 0;
  long base = (long)tile - 1;
  long spins = 0;
  const u32 ep = epoch & 0x3fffffffu;
  for (;;) {
    long idx = base - lane;
    u32 flag, val;
    if (idx >= 0) {
      u64 s = ld_volatile(&status[idx]);
      bool fresh = (u32)(s >> 34) == ep;
      flag = fresh ? (u32)((s >> 32) & 3u) : 0u;
      val = (u32)s;
    } else {
      flag = ST_INC;
      val = 0;
    }
    unsigned inc = __ballot_sync(FULL, flag == ST_INC);
    unsigned inv = __ballot_sync(FULL, flag == 0);
    unsigned need = inc ? ((inc & (0u - inc)) << 1) - 1 : FULL;  // lanes up to the nearest inclusive
    if (inv & need) {
      if (++spins > LOOKBACK_SPIN_LIMIT) {
        if (lane == 0) atomicOr(&ctl->error, ERR_LOOKBACK_TIMEOUT);
        break;
      }
      __nanosleep(64);
      continue;
    }
    u32 v = ((need >> lane) & 1u) ? val : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    excl += v;
    if (inc) break;
    base -= 32;
  }
  if (lane == 0) st_volatile(&status[tile], pack_status(epoch, ST_INC, excl + agg));
  return excl;
}

template <int W>
__device__ __forceinline__ void load_key(const u64* __restrict__ keys, u64 row, u64* k) {
  const u64* p = keys + row * W;
  if constexpr (W % 2 == 0) {
#pragma unroll
    for (int i = 0; i < W; i += 2) {
      ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(p + i));
      k[i] = v.x;
      k[i + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < W; ++i) k[i] = __ldg(p + i);
  }
}
template <int W>
__device__ __forceinline__ void store_key(u64* keys, u64 row, const u64* k) {
  u64* p = keys + row * W;
  if constexpr (W % 2 == 0) {
#pragma unroll
    for (int i = 0; i < W; i += 2) *reinterpret_cast<ulonglong2*>(p + i) = make_ulonglong2(k[i], k[i + 1]);
  } else {
#pragma unroll
    for (int i = 0; i < W; ++i) p[i] = k[i];
  }
}

// Row holding key q among rows < n_pre, or -1.  Rows inserted by the running
// gate (>= n_pre) are skipped: no lookup of this gate can target them.
template <int W>
__device__ long long lookup(const u64* q, u64 n_pre, const u64* __restrict__ keys, const u64* table,
                            u64 mask, Ctl* ctl) {
  const u64 h = key_hash<W>(q);
  const u32 fp = (u32)(h >> 32);
  u64 i = h & mask;
  for (u64 probe = 0; probe <= mask; ++probe) {
    const u64 s = __ldcg(table + i);
    if (s == EMPTY_SLOT) return -1;
    const u32 row = (u32)s;
    if ((u32)(s >> 32) == fp && row < n_pre) {
      const u64* kp = keys + (u64)row * W;
      bool eq = true;
#pragma unroll
      for (int w = 0; w < W; ++w) eq &= __ldg(kp + w) == q[w];
      if (eq) return row;
    }
    i = (i + 1) & mask;
  }
  atomicOr(&ctl->error, ERR_PROBE_OVERFLOW);
  return -1;
}

template <int W>
__device__ void insert(const u64* q, u64 row, u64* table, u64 mask, Ctl* ctl) {
  const u64 h = key_hash<W>(q);
  const u64 v = ((h >> 32) << 32) | (row & 0xffffffffULL);
  u64 i = h & mask;
  for (u64 probe = 0; probe <= mask; ++probe) {
    if (__ldcg(table + i) == EMPTY_SLOT && atomicCAS(table + i, EMPTY_SLOT, v) == EMPTY_SLOT) return;
    i = (i + 1) & mask;
  }
  atomicOr(&ctl->error, ERR_PROBE_OVERFLOW);
}

// -(Im phase) of G*K = i^p * sign: the sin-branch multiplier (coeff.rs:151-168).
__device__ __forceinline__ double neg_im(int p, double sign) {
  return p == 1 ? -sign : (p == 3 ? sign : 0.0);
}

template <class Ops>
struct OpsOf;

template <int ALG>
struct Alg;
template <>
struct Alg<0> {
  using T = PauliOps;
};
template <>
struct Alg<1> {
  using T = MajoranaOps;
};

// Shared-memory block used by every compaction kernel.
struct TileSmem {
  u32 tile;
  u32 excl;
  u32 cnt[32];  // item-major per-warp counts, then their exclusive prefixes
};

// Entry: decide (uniformly for the whole grid) whether this op runs.
__device__ __forceinline__ void op_entry(Ctl* ctl, u64 cap_needed, u64 cap, u32 op, u64* n_out, u32* par_out,
                                         u32* epoch_out, bool* skip_out) {
  const u32 par = *(volatile u32*)&ctl->parity;
  const u64 n = *(volatile u64*)&ctl->n[par];
  const u32 halt = *(volatile u32*)&ctl->halt;
  bool skip = halt != NOT_HALTED;
  if (!skip && cap_needed > cap) {
    skip = true;
    if (threadIdx.x == 0) atomicMin(&ctl->halt, op);
  }
  *n_out = n;
  *par_out = par;
  *epoch_out = *(volatile u32*)&ctl->epoch;
  *skip_out = skip;
}

// Exit: the last block out publishes the new count and resets the protocol.
__device__ __forceinline__ void op_exit(Ctl* ctl, u64* hist, u32 op, bool skip, bool changes_n, u32 par,
                                        u64 n_in, u32 ntiles, u32 epoch) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const u32 d = atomicAdd(&ctl->done, 1u);
    if (d == gridDim.x - 1) {
      __threadfence();
      u64 n_new = n_in;
      if (!skip && changes_n) {
        n_new = ntiles ? *(volatile u64*)&ctl->n_next : n_in;
        ctl->n[par ^ 1u] = n_new;
        ctl->parity = par ^ 1u;
      }
      if (!skip) {
        if (hist) hist[op] = n_new;
        if (n_new > ctl->peak) ctl->peak = n_new;
      }
      ctl->ticket = 0;
      ctl->done = 0;
      ctl->epoch = epoch + 1;
      __threadfence();
    }
  }
}

__device__ __forceinline__ u32 next_tile(Ctl* ctl, TileSmem& sm) {
  if (threadIdx.x == 0) sm.tile = atomicAdd(&ctl->ticket, 1u);
  __syncthreads();
  const u32 t = sm.tile;
  return t;
}

// Item-major block scan of ITEMS emit flags per thread + look-back.
// Returns the per-item exclusive rank base for this warp in sm.cnt and the
// tile's global exclusive prefix in sm.excl.
__device__ __forceinline__ void tile_scan(u32 emit_mask, unsigned* masks, TileSmem& sm, u64* status, u32 t,
                                          u32 ntiles, u64 n_base, u32 epoch, Ctl* ctl) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    masks[k] = __ballot_sync(FULL, (emit_mask >> k) & 1u);
    if (lane == 0) sm.cnt[k * NWARPS + warp] = __popc(masks[k]);
  }
  __syncthreads();
  if (warp == 0) {
    u32 v = sm.cnt[lane];
    u32 inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      u32 y = __shfl_up_sync(FULL, inc, o);
      if (lane >= o) inc += y;
    }
    sm.cnt[lane] = inc - v;
    const u32 agg = __shfl_sync(FULL, inc, 31);
    const u32 excl = lookback(status, t, agg, epoch, ctl);
    if (lane == 0) {
      sm.excl = excl;
      if (t == ntiles - 1) *(volatile u64*)&ctl->n_next = n_base + excl + agg;
    }
  }
  __syncthreads();
}

// ------------------------------------------------------------------ gate
template <int W, int ALG>
__global__ void __launch_bounds__(BLOCK) gate_kernel(const GateArgs<W> a, const DevBufs b) {
  using Ops = typename Alg<ALG>::T;
  __shared__ TileSmem sm;
  Ctl* ctl = b.ctl;
  u64 N;
  u32 par, epoch;
  bool skip;
  op_entry(ctl, 0, 0, a.op, &N, &par, &epoch, &skip);
  // Children this gate can create are at most the anticommuting rows, so
  // 2N rows must fit before the gate may start.
  if (!skip && 2 * N > b.cap) {
    skip = true;
    if (threadIdx.x == 0) atomicMin(&ctl->halt, a.op);
  }
  const u32 ntiles = (u32)((N + TILE - 1) / TILE);
  if (!skip) {
    // TermBudget: below the floor, every lossy predicate is off (termsum.rs:60-76).
    const bool lossless = a.min_terms && N < a.min_terms;
    const u32 wcut = lossless ? NO_WEIGHT_CUT : a.max_weight;
    const bool ccut = !lossless && a.has_min_coeff;
    const double minc = a.min_coeff;
    const double sn = a.sn, cs = a.cs;
    // Emit state of a source with coefficient c, branch b and child key ch
    // (termsum.rs:701-751): HELD by the magnitude precheck, DROP by weight,
    // else EMIT.
    auto state = [&](double c, const u64* ch) -> int {
      if (ccut && fabs(c * sn) < minc) return S_HELD;
      if (wcut != NO_WEIGHT_CUT && Ops::template weight<W>(ch, a.n_units) > wcut) return S_DROP;
      return S_EMIT;
    };
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u32 n_anti = 0;
    for (;;) {
      const u32 t = next_tile(ctl, sm);
      if (t >= ntiles) break;
      u32 emit_mask = 0;
      double bval[ITEMS];
#pragma unroll
      for (int k = 0; k < ITEMS; ++k) {
        bval[k] = 0.0;
        const u64 r = (u64)t * TILE + (u64)k * BLOCK + threadIdx.x;
        if (r >= N) continue;
        u64 key[W];
        load_key<W>(b.keys, r, key);
        if (!Ops::template anticommutes<W>(a.g, key)) continue;
        ++n_anti;
        u64 q[W];
#pragma unroll
        for (int w = 0; w < W; ++w) q[w] = key[w] ^ a.g.gen[w];
        const long long j = lookup<W>(q, N, b.keys, b.table, b.table_mask, ctl);
        if (j >= 0 && (u64)j < r) continue;  // the lower row of the pair owns it
        const double c = b.coeffs[r];
        const double bi = (c * sn) * neg_im(Ops::template product_exp<W>(a.g, key), a.g.sign);
        const int si = state(c, q);
        if (j < 0) {
          b.coeffs[r] = c * cs;
          if (si == S_EMIT) {
            emit_mask |= 1u << k;
            bval[k] = bi;
          }
        } else {
          const double cj = b.coeffs[j];
          const double bj = (cj * sn) * neg_im(Ops::template product_exp<W>(a.g, q), a.g.sign);
          const int sj = state(cj, key);
          const bool to_j = si == S_EMIT || (si == S_HELD && sj == S_EMIT);
          const bool to_i = sj == S_EMIT || (sj == S_HELD && si == S_EMIT);
          double ni = c * cs;
          if (to_i) ni = ni + bj;
          double nj = cj * cs;
          if (to_j) nj = nj + bi;
          b.coeffs[r] = ni;
          b.coeffs[j] = nj;
        }
      }
      unsigned masks[ITEMS];
      tile_scan(emit_mask, masks, sm, b.status, t, ntiles, N, epoch, ctl);
      const unsigned lt = (1u << lane) - 1u;
#pragma unroll
      for (int k = 0; k < ITEMS; ++k) {
        if (!((emit_mask >> k) & 1u)) continue;
        const u64 r = (u64)t * TILE + (u64)k * BLOCK + threadIdx.x;
        const u64 row = N + sm.excl + sm.cnt[k * NWARPS + warp] + __popc(masks[k] & lt);
        if (row >= b.cap) {
          atomicOr(&ctl->error, ERR_CAPACITY);
          continue;
        }
        u64 q[W];
        load_key<W>(b.keys, r, q);
#pragma unroll
        for (int w = 0; w < W; ++w) q[w] ^= a.g.gen[w];
        store_key<W>(b.keys, row, q);
        b.coeffs[row] = bval[k];
        insert<W>(q, row, b.table, b.table_mask, ctl);
      }
      __syncthreads();
    }
    // per-op count of anticommuting rows (one atomic per warp)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_anti += __shfl_xor_sync(FULL, n_anti, o);
    if (lane == 0 && n_anti && b.anti) atomicAdd(b.anti + a.op, (u64)n_anti);
  }
  op_exit(ctl, b.hist, a.op, skip, true, par, N, ntiles, epoch);
}

// A rotation with |sin| < 1e-9 only scales the anticommuting rows by cos
// (partitioned_termsum.rs:303-308, termsum.rs:551-557).
template <int W, int ALG>
__global__ void __launch_bounds__(BLOCK) phase_only_kernel(const GateArgs<W> a, const DevBufs b) {
  using Ops = typename Alg<ALG>::T;
  __shared__ TileSmem sm;
  Ctl* ctl = b.ctl;
  u64 N;
  u32 par, epoch;
  bool skip;
  op_entry(ctl, 0, 0, a.op, &N, &par, &epoch, &skip);
  const u32 ntiles = (u32)((N + TILE - 1) / TILE);
  if (!skip) {
    for (;;) {
      const u32 t = next_tile(ctl, sm);
      if (t >= ntiles) break;
#pragma unroll
      for (int k = 0; k < ITEMS; ++k) {
        const u64 r = (u64)t * TILE + (u64)k * BLOCK + threadIdx.x;
        if (r >= N) continue;
        u64 key[W];
        load_key<W>(b.keys, r, key);
        if (Ops::template anticommutes<W>(a.g, key)) b.coeffs[r] *= a.cs;
      }
      __syncthreads();
    }
  }
  op_exit(ctl, b.hist, a.op, skip, false, par, N, ntiles, epoch);
}

// ----------------------------------------------------------------- noise
// One noisy layer: c *= factor[min(w, len-1)] (engine.rs:119-125), then the
// reclaim keeps weight <= cut and |c| >= cut (termsum.rs:472-497,
// partitioned_termsum.rs:581-608), compacting survivors in row order into
// the alternate buffers and re-inserting them into the (cleared) table.
template <int W, int ALG>
__global__ void __launch_bounds__(BLOCK) noise_kernel(const NoiseArgs a, const DevBufs b) {
  using Ops = typename Alg<ALG>::T;
  __shared__ TileSmem sm;
  Ctl* ctl = b.ctl;
  u64 N;
  u32 par, epoch;
  bool skip;
  op_entry(ctl, 0, 0, a.op, &N, &par, &epoch, &skip);
  const u32 ntiles = (u32)((N + TILE - 1) / TILE);
  if (!skip) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const u32 last = a.table_len - 1;
    for (;;) {
      const u32 t = next_tile(ctl, sm);
      if (t >= ntiles) break;
      u32 keep_mask = 0;
      double cv[ITEMS];
#pragma unroll
      for (int k = 0; k < ITEMS; ++k) {
        cv[k] = 0.0;
        const u64 r = (u64)t * TILE + (u64)k * BLOCK + threadIdx.x;
        if (r >= N) continue;
        u64 key[W];
        load_key<W>(b.keys, r, key);
        const u32 w = Ops::template weight<W>(key, a.n_units);
        const double c = b.coeffs[r] * __ldg(a.factors + (w < last ? w : last));
        if (!a.compact) {
          b.coeffs[r] = c;
          continue;
        }
        cv[k] = c;
        const bool keep = (a.max_weight == NO_WEIGHT_CUT || w <= a.max_weight) &&
                          (!a.has_min_coeff || fabs(c) >= a.min_coeff);
        keep_mask |= (u32)keep << k;
      }
      if (a.compact) {
        unsigned masks[ITEMS];
        tile_scan(keep_mask, masks, sm, b.status, t, ntiles, 0, epoch, ctl);
        const unsigned lt = (1u << lane) - 1u;
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
          if (!((keep_mask >> k) & 1u)) continue;
          const u64 r = (u64)t * TILE + (u64)k * BLOCK + threadIdx.x;
          const u64 row = sm.excl + sm.cnt[k * NWARPS + warp] + __popc(masks[k] & lt);
          u64 key[W];
          load_key<W>(b.keys, r, key);
          store_key<W>(b.keys_alt, row, key);
          b.coeffs_alt[row] = cv[k];
          insert<W>(key, row, b.table, b.table_mask, ctl);
        }
      }
      __syncthreads();
    }
  }
  op_exit(ctl, b.hist, a.op, skip, a.compact != 0, par, N, ntiles, epoch);
}

// ------------------------------------------------------------ expectation
// Generic phase exponent of gen*key for a raw generator (used by the frame
// conjugation, where every tableau row acts as a generator).
template <int W, int ALG>
__device__ int product_exp_raw(const u64* gen, const u64* key) {
  if constexpr (ALG == 0) {
    int yg = 0, yk = 0, yo = 0, zx = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) {
      u64 o = key[i] ^ gen[i];
      yg += __popcll(gen[i] & (gen[i] >> 1) & EVEN);
      yk += __popcll(key[i] & (key[i] >> 1) & EVEN);
      yo += __popcll(o & (o >> 1) & EVEN);
      zx += __popcll((gen[i] >> 1) & key[i] & EVEN);
    }
    return (yg + yk - yo + 2 * zx) & 3;
  } else {
    int lg = 0, lk = 0, lo = 0, sw = 0;
    u32 above = 0;  // parity of gen modes in higher words
#pragma unroll
    for (int i = W - 1; i >= 0; --i) {
      u64 o = key[i] ^ gen[i];
      int pg = __popcll(gen[i]), pk = __popcll(key[i]);
      lg += pg;
      lk += pk;
      lo += __popcll(o);
      u64 s = gen[i] >> 1;
      s ^= s >> 1;
      s ^= s >> 2;
      s ^= s >> 4;
      s ^= s >> 8;
      s ^= s >> 16;
      s ^= s >> 32;
      sw ^= (__popcll(key[i] & s) & 1) ^ (pk & (int)above);
      above ^= (u32)(pg & 1);
    }
    auto herm = [](int l) { return ((l & 3) >= 2) ? 1 : 0; };
    return (herm(lg) + herm(lk) - herm(lo) + 2 * (sw & 1)) & 3;
  }
}

// Readout conjugation through a deferred Clifford frame
// (tableau.rs:93-143): fold the rows selected by the key's bits, tracking the
// phase of the rebuilt source and of the image; the sign is -1 iff their
// ratio is -1.
template <int W, int ALG>
__device__ double conjugate_key(const u64* key, const u64* images, const int* signs, u32 rows, u64* out) {
  u64 src[W];
#pragma unroll
  for (int i = 0; i < W; ++i) src[i] = out[i] = 0;
  int se = 0, ie = 0;
#pragma unroll
  for (int wi = 0; wi < W; ++wi) {
    u64 bits = key[wi];
    while (bits) {
      const int bpos = __ffsll((long long)bits) - 1;
      bits &= bits - 1;
      const u32 p = (u32)(wi * 64 + bpos);
      if (p >= rows) continue;
      u64 e[W];
#pragma unroll
      for (int i = 0; i < W; ++i) e[i] = 0;
      e[wi] = 1ULL << bpos;
      se += product_exp_raw<W, ALG>(e, src);
      src[wi] ^= e[wi];
      const u64* img = images + (u64)p * W;
      u64 g[W];
#pragma unroll
      for (int i = 0; i < W; ++i) g[i] = __ldg(img + i);
      ie += product_exp_raw<W, ALG>(g, out) + (signs[p] < 0 ? 2 : 0);
#pragma unroll
      for (int i = 0; i < W; ++i) out[i] ^= g[i];
    }
  }
  return (((ie - se) & 3) == 2) ? -1.0 : 1.0;
}

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
__device__ __forceinline__ void dd_add(double& hi, double& lo, double v) {
  double s, e;
  two_sum(hi, v, s, e);
  e += lo;
  two_sum(s, e, hi, lo);
}

// sum c * <s|frame(K)|s> in double-double, plus the count of |c| < min_coeff
// (partitioned_termsum.rs:611-697).
template <int W, int ALG>
__global__ void __launch_bounds__(BLOCK) expect_kernel(const ExpectArgs a, const DevBufs b,
                                                       ExpectPartial* partials) {
  using Ops = typename Alg<ALG>::T;
  const u64 N = b.ctl->n[b.ctl->parity];
  double hi = 0, lo = 0, ab = 0;
  u64 below = 0;
  for (u64 r = (u64)blockIdx.x * BLOCK + threadIdx.x; r < N; r += (u64)gridDim.x * BLOCK) {
    u64 key[W];
    load_key<W>(b.keys, r, key);
    const double c = b.coeffs[r];
    if (a.has_min_coeff && fabs(c) < a.min_coeff) ++below;
    double v;
    if (a.frame_images) {
      u64 img[W];
      const double sg = conjugate_key<W, ALG>(key, a.frame_images, a.frame_signs, a.frame_rows, img);
      v = c * sg * Ops::template trace<W>(img, a.state, a.n_units);
    } else {
      v = c * Ops::template trace<W>(key, a.state, a.n_units);
    }
    if (v != 0.0) {
      dd_add(hi, lo, v);
      ab += fabs(v);
    }
  }
  // warp then block reduction (double-double)
  for (int o = 16; o > 0; o >>= 1) {
    double ohi = __shfl_xor_sync(FULL, hi, o), olo = __shfl_xor_sync(FULL, lo, o);
    dd_add(hi, lo, ohi);
    dd_add(hi, lo, olo);
    ab += __shfl_xor_sync(FULL, ab, o);
    below += __shfl_xor_sync(FULL, below, o);
  }
  __shared__ double shi[NWARPS], slo[NWARPS], sab[NWARPS];
  __shared__ u64 sbl[NWARPS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    shi[warp] = hi;
    slo[warp] = lo;
    sab[warp] = ab;
    sbl[warp] = below;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double h = 0, l = 0, s = 0;
    u64 bl = 0;
    for (int w = 0; w < NWARPS; ++w) {
      dd_add(h, l, shi[w]);
      dd_add(h, l, slo[w]);
      s += sab[w];
      bl += sbl[w];
    }
    partials[blockIdx.x] = ExpectPartial{h, l, s, bl};
  }
}

// Re-inserts rows [0, N) into a cleared table (after a capacity change).
template <int W>
__global__ void rebuild_kernel(const DevBufs b) {
  const u64 N = b.ctl->n[b.ctl->parity];
  for (u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (u64)gridDim.x * blockDim.x) {
    u64 key[W];
    load_key<W>(b.keys, r, key);
    insert<W>(key, r, b.table, b.table_mask, b.ctl);
  }
}

// Final terms through the readout frame, sign folded into the coefficient.
template <int W, int ALG>
__global__ void conjugate_kernel(const DevBufs b, const u64* images, const int* signs, u32 rows, u64* out_keys,
                                 double* out_coeffs, u64 n) {
  for (u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (u64)gridDim.x * blockDim.x) {
    u64 key[W], img[W];
    load_key<W>(b.keys, r, key);
    const double sg = conjugate_key<W, ALG>(key, images, signs, rows, img);
    store_key<W>(out_keys, r, img);
    out_coeffs[r] = b.coeffs[r] * sg;
  }
}

}  // namespace

int launch_blocks() {
  static int cached = 0;
  if (cached) return cached;
  int dev = 0, sms = 148, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gate_kernel<4, 0>, BLOCK, 0);
  if (per_sm < 1) per_sm = 1;
  cached = sms * per_sm;
  return cached;
}

template <int W, int ALG>
cudaError_t launch_gate(const GateArgs<W>& a, const DevBufs& b, int grid, cudaStream_t s) {
  gate_kernel<W, ALG><<<grid, BLOCK, 0, s>>>(a, b);
  return cudaGetLastError();
}
template <int W, int ALG>
cudaError_t launch_phase_only(const GateArgs<W>& a, const DevBufs& b, int grid, cudaStream_t s) {
  phase_only_kernel<W, ALG><<<grid, BLOCK, 0, s>>>(a, b);
  return cudaGetLastError();
}
template <int W, int ALG>
cudaError_t launch_noise(const NoiseArgs& a, const DevBufs& b, int grid, cudaStream_t s) {
  noise_kernel<W, ALG><<<grid, BLOCK, 0, s>>>(a, b);
  return cudaGetLastError();
}
template <int W, int ALG>
cudaError_t launch_expect(const ExpectArgs& a, const DevBufs& b, ExpectPartial* partials, int grid,
                          cudaStream_t s) {
  expect_kernel<W, ALG><<<grid, BLOCK, 0, s>>>(a, b, partials);
  return cudaGetLastError();
}
template <int W>
cudaError_t launch_rebuild(const DevBufs& b, int grid, cudaStream_t s) {
  rebuild_kernel<W><<<grid, 256, 0, s>>>(b);
  return cudaGetLastError();
}
template <int W>
cudaError_t launch_conjugate(const DevBufs& b, const u64* images, const int* signs, u32 rows, int alg,
                             u64* out_keys, double* out_coeffs, u64 n, cudaStream_t s) {
  const int grid = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
  if (grid == 0) return cudaSuccess;
  if (alg == 0)
    conjugate_kernel<W, 0><<<grid, 256, 0, s>>>(b, images, signs, rows, out_keys, out_coeffs, n);
  else
    conjugate_kernel<W, 1><<<grid, 256, 0, s>>>(b, images, signs, rows, out_keys, out_coeffs, n);
  return cudaGetLastError();
}

#define PQ_INSTANTIATE(Wv, Av)                                                                         \
  template cudaError_t launch_gate<Wv, Av>(const GateArgs<Wv>&, const DevBufs&, int, cudaStream_t);       \
  template cudaError_t launch_phase_only<Wv, Av>(const GateArgs<Wv>&, const DevBufs&, int, cudaStream_t); \
  template cudaError_t launch_noise<Wv, Av>(const NoiseArgs&, const DevBufs&, int, cudaStream_t);         \
  template cudaError_t launch_expect<Wv, Av>(const ExpectArgs&, const DevBufs&, ExpectPartial*, int,      \
                                             cudaStream_t);
#define PQ_INSTANTIATE_W(Wv)                                                                            \
  PQ_INSTANTIATE(Wv, 0)                                                                                 \
  PQ_INSTANTIATE(Wv, 1)                                                                                 \
  template cudaError_t launch_rebuild<Wv>(const DevBufs&, int, cudaStream_t);                           \
  template cudaError_t launch_conjugate<Wv>(const DevBufs&, const u64*, const int*, u32, int, u64*, double*, \
                                            u64, cudaStream_t);

PQ_INSTANTIATE_W(1)
PQ_INSTANTIATE_W(2)
PQ_INSTANTIATE_W(4)
PQ_INSTANTIATE_W(8)

}  // namespace pq
