// pq_kernels.cu -- the hot path of the B200 propagation engine.
//
// The whole op sequence of a propagation (noise layers and gates, in
// Heisenberg order) runs as ONE cooperative persistent kernel, sweep_kernel.
// Its blocks are co-resident; a bounded grid barrier separates consecutive
// ops, so a gate costs no launch.  Per gate the kernel replaces the
// reference's scan -> route -> absorb -> claim -> rescue rounds
// (crates/core/src/engine/partitioned_termsum.rs:276-450,
//  crates/core/src/engine/termsum.rs:561-800) with a single pass:
//
//   * each row is tested for anticommutation by popcount parity;
//   * an anticommuting row looks its child K = G.S up in the open-addressing
//     hash table (pre-gate rows only).  K -> G.K is an involution, so a row
//     has at most one partner; the lower row of a pair owns both
//     coefficients and applies the pair rule to both from the pre-gate
//     values, so no coefficient is ever written by two threads;
//   * a lone row whose branch survives the emit cutoff creates its child;
//     children are appended in row order through a warp-ballot / block scan
//     and a decoupled look-back across tiles, and inserted into the table by
//     atomicCAS on the packed (fingerprint, row) slot.
//
// Rows are never removed by a gate.  A noisy layer damps every row; with a
// truncation configured it then clears the table, filters the rows, compacts
// the survivors in row order into the other row buffer and re-inserts them
// (termsum.rs:472-497).
//
// Before each gate the kernel checks that twice the live count fits the row
// capacity (a gate appends at most one child per row).  If it does not, every
// block stops at that op and the host grows the buffers and relaunches from
// it.  Every spin-wait is bounded and raises an error bit instead of hanging.
#include <cuda_runtime.h>

#include <cstdio>

#include "pq_kernels.cuh"

namespace pq {

namespace {

constexpr int BLOCK = 256;
constexpr int NWARPS = BLOCK / 32;
constexpr int MAX_ITEMS = 4;  // rows per thread per tile; items * NWARPS <= 32
static_assert(MAX_ITEMS * NWARPS <= 32, "tile scan uses one warp");

constexpr u32 ST_AGG = 1u, ST_INC = 2u;
constexpr unsigned FULL = 0xffffffffu;
constexpr u32 BAR_GROUPS = SweepState::BAR_GROUPS;
// A fused op runs both rotations in one pass while each block has at most
// this many tiles of rows; above, one after the other.
constexpr u32 GATE2_TILES_PER_BLOCK = 4;
static_assert(GROUP_MAX == 2, "the sweep runs fused pairs (gate2_tiles)");

enum : int { S_EMIT = 0, S_HELD = 1, S_DROP = 2 };

__device__ __forceinline__ u64 pack_status(u32 epoch, u32 flag, u32 value) {
  return ((u64)(epoch & 0x3fffffffu) << 34) | ((u64)flag << 32) | value;
}
__device__ __forceinline__ u64 ld_volatile(const u64* p) { return *(const volatile u64*)p; }
__device__ __forceinline__ void st_volatile(u64* p, u64 v) { *(volatile u64*)p = v; }

// The blocks running one propagation: `bid` of `nblk` (the whole grid for a
// single run, a contiguous slice of it for one instance of a batch).
struct Grp {
  u32 bid, nblk;
};

// Grid barrier (sense by generation).  Above BAR_FLAT blocks it is two-level:
// each block arrives on one of BAR_GROUPS counters (each on its own 128-byte
// line), the last arrival of a group arrives on the top counter; smaller grids
// arrive on the top counter directly.  The last top arrival releases
// everyone by bumping the generation.  Every wait is bounded; once one
// expires, ERR_BARRIER_TIMEOUT makes every later barrier fall through.
// The three steps run on thread 0 of each block, after the block's
// __syncthreads; the arrivals are release-acquire atomics at GPU scope and
// the wait an acquire load, so what any thread of any block wrote before the
// barrier is visible to every thread after it, without a full fence.
__device__ __forceinline__ u32 atom_add_acq_rel(u32* p, u32 v) {
  u32 old;
  asm volatile("atom.add.acq_rel.gpu.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ u32 ld_acquire(const u32* p) {
  u32 v;
  asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(u32* p, u32 v) {
  asm volatile("st.release.gpu.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Arrives; true for the last arrival of the whole grid.  Grids of up to
// BAR_FLAT blocks arrive on the top counter directly: one atomic round trip
// instead of two, for at most BAR_FLAT atomics queued on one address.
constexpr u32 BAR_FLAT = 320;
__device__ __forceinline__ bool barrier_arrive(SweepState* st, const Grp g_) {
  const u32 nb = g_.nblk;
  if (nb <= BAR_FLAT) return atom_add_acq_rel(&st->bar_count, 1u) == nb - 1;
  const u32 grp = g_.bid % BAR_GROUPS;
  const u32 in_grp = nb / BAR_GROUPS + (grp < nb % BAR_GROUPS ? 1u : 0u);
  const u32 n_grp = nb < BAR_GROUPS ? nb : BAR_GROUPS;
  if (atom_add_acq_rel(&st->bar_group[grp].count, 1u) != in_grp - 1) return false;
  st->bar_group[grp].count = 0;  // no block arrives on it again before the release
  return atom_add_acq_rel(&st->bar_count, 1u) == n_grp - 1;
}
__device__ __forceinline__ void barrier_release(SweepState* st, u32 g) {
  st->bar_count = 0;
  st_release(&st->bar_gen, g + 1);  // orders the two resets and everything before it
}
__device__ __forceinline__ void barrier_wait(SweepState* st, u32 g) {
  const u32 limit = st->barrier_limit;  // set by the host for the launch
  u32 spins = 0;
  while (ld_acquire(&st->bar_gen) == g) {
    if (*(volatile u32*)&st->error & ERR_BARRIER_TIMEOUT) break;
    if (++spins > limit) {
      atomicOr(&st->error, ERR_BARRIER_TIMEOUT);
      break;
    }
    __nanosleep(20);
  }
}

__device__ __forceinline__ void grid_barrier(SweepState* st, u32& gen, const Grp g_) {
  __syncthreads();
  if (threadIdx.x == 0) {
    if (barrier_arrive(st, g_))
      barrier_release(st, gen);
    else
      barrier_wait(st, gen);
    ++gen;
  }
  __syncthreads();
}

// What every block needs after the end-of-op barrier, read once by thread 0.
struct OpShared {
  u64 n;            // live rows entering the next op
  u32 err;          // SweepState::error
  u32 yield_after;  // SweepState::yield_after
  u32 extra[3];     // words the op asked for (a fused op's rows created by each rotation)
};

// The barrier between two ops of a sweep.  Thread 0 of each block, once it
// has arrived (or released), runs prefetch() -- loading the next op's
// descriptors, which do not depend on this op, while it waits -- and after
// the release reads the next op's live count and the error / yield words
// together into shared memory, one round trip for the block.
template <class Prefetch>
__device__ __forceinline__ void op_barrier(SweepState* st, u32& gen, const Grp g_, const u64* n_next, const u32* extra,
                                           u32 n_extra, OpShared& os, Prefetch prefetch) {
  __syncthreads();
  if (threadIdx.x == 0) {
    if (barrier_arrive(st, g_)) {
      barrier_release(st, gen);
      prefetch();
    } else {
      prefetch();
      barrier_wait(st, gen);
    }
    ++gen;
    const u64 n = ld_volatile(n_next);
    const u32 e = *(volatile u32*)&st->error;
    const u32 y = *(volatile u32*)&st->yield_after;
    u32 x[3] = {0u, 0u, 0u};
    if (extra)
      for (u32 i = 0; i < n_extra && i < 3; ++i) x[i] = *(const volatile u32*)(extra + i);
    os.n = n;
    os.err = e;
    os.yield_after = y;
    for (int i = 0; i < 3; ++i) os.extra[i] = x[i];
  }
  __syncthreads();
}

// Decoupled look-back (called by all lanes of warp 0): publishes this tile's
// aggregate, walks predecessors 32 at a time, returns the exclusive prefix.
__device__ u32 lookback(u64* status, u32 tile, u32 agg, u32 epoch, SweepState* st) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) st_volatile(&status[0], pack_status(epoch, ST_INC, agg));
    return 0;
  }
  if (lane == 0) st_volatile(&status[tile], pack_status(epoch, ST_AGG, agg));
  u32 excl = 0;
  long base = (long)tile - 1;
  const u32 limit = st->lookback_limit;  // set by the host for the launch
  u32 spins = 0;
  const u32 ep = epoch & 0x3fffffffu;
  for (;;) {
    const long idx = base - lane;
    u32 flag, val;
    if (idx >= 0) {
      const u64 s = ld_volatile(&status[idx]);
      flag = ((u32)(s >> 34) == ep) ? (u32)((s >> 32) & 3u) : 0u;
      val = (u32)s;
    } else {
      flag = ST_INC;
      val = 0;
    }
    const unsigned inc = __ballot_sync(FULL, flag == ST_INC);
    const unsigned inv = __ballot_sync(FULL, flag == 0);
    const unsigned need = inc ? ((inc & (0u - inc)) << 1) - 1 : FULL;  // lanes up to the nearest inclusive
    if (inv & need) {
      if (++spins > limit) {
        if (lane == 0) atomicOr(&st->error, ERR_LOOKBACK_TIMEOUT);
        break;
      }
      __nanosleep(32);
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
__device__ __forceinline__ void load_key(const u64* keys, u64 row, u64* k) {
  const u64* p = keys + row * W;
  if constexpr (W % 2 == 0) {
#pragma unroll
    for (int i = 0; i < W; i += 2) {
      const ulonglong2 v = __ldcg(reinterpret_cast<const ulonglong2*>(p + i));
      k[i] = v.x;
      k[i + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < W; ++i) k[i] = __ldcg(p + i);
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

// The table is linear-probed from a bucket of 2, 4 or 8 slots (bmask = ~(slots
// - 1); 4 slots are one 32-byte sector): a lookup starts at the first slot of
// the key's bucket and scans forward until it meets the key or an empty slot;
// an insert takes the first empty slot of the same sequence.  The first probe
// loads 4 slots, so a bucket of 2 may span two sectors and one of 8 takes two
// probes when its first half is full.
__device__ __forceinline__ u64 bucket_start(u64 h, u64 mask, u64 bmask) { return (h & mask) & bmask; }

// Continues a lookup of q from slot i (see bucket_start).  Rows the running
// gate appends (>= n_pre) are skipped: no lookup of this gate can target them.
template <int W>
__device__ long long lookup_from(const u64* q, u32 fp, u64 i, u64 n_pre, const u64* keys, const u64* table,
                                 u64 mask, SweepState* st) {
  for (u64 probe = 0; probe <= mask; ++probe) {
    const u64 s = __ldcg(table + i);
    if (s == EMPTY_SLOT) return -1;
    const u32 row = (u32)s;
    if ((u32)(s >> 32) == fp && row < n_pre) {
      const u64* kp = keys + (u64)row * W;
      bool eq = true;
#pragma unroll
      for (int w = 0; w < W; ++w) eq &= __ldcg(kp + w) == q[w];
      if (eq) return row;
    }
    i = (i + 1) & mask;
  }
  atomicOr(&st->error, ERR_PROBE_OVERFLOW);
  return -1;
}

template <int W>
__device__ void insert(const u64* q, u64 row, u64* table, u64 mask, u64 bmask, u32* error) {
  const u64 h = key_hash<W>(q);
  const u64 v = ((h >> 32) << 32) | (row & 0xffffffffULL);
  u64 i = bucket_start(h, mask, bmask);
  for (u64 probe = 0; probe <= mask; ++probe) {
    if (__ldcg(table + i) == EMPTY_SLOT && atomicCAS(table + i, EMPTY_SLOT, v) == EMPTY_SLOT) return;
    i = (i + 1) & mask;
  }
  atomicOr(error, ERR_PROBE_OVERFLOW);
}

// Claims a slot for q before its row is known: the slot holds q's
// fingerprint and the placeholder row PENDING_ROW (never below a lookup's
// n_pre, so no lookup of the running op can match it) until set_row writes
// the row into its low half.  Claiming early lets the atomic round trip
// overlap the tile scan.  Returns the slot, or NO_SLOT if the table is full.
constexpr u32 PENDING_ROW = 0xfffffffeu;
constexpr u64 NO_SLOT = ~0ULL;
template <int W>
__device__ u64 claim_slot(const u64* q, u64* table, u64 mask, u64 bmask, u32* error) {
  const u64 h = key_hash<W>(q);
  const u64 v = ((h >> 32) << 32) | PENDING_ROW;
  u64 i = bucket_start(h, mask, bmask);
  for (u64 probe = 0; probe <= mask; ++probe) {
    if (__ldcg(table + i) == EMPTY_SLOT && atomicCAS(table + i, EMPTY_SLOT, v) == EMPTY_SLOT) return i;
    i = (i + 1) & mask;
  }
  atomicOr(error, ERR_PROBE_OVERFLOW);
  return NO_SLOT;
}
__device__ __forceinline__ void set_row(u64* table, u64 slot, u64 row) {
  if (slot != NO_SLOT) reinterpret_cast<u32*>(table + slot)[0] = (u32)row;  // little-endian low half
}

// Row holding q among the pre-gate rows, or -1: the key's first bucket is
// one 32-byte load, so most lookups finish with it (plus the candidate row's
// key on a fingerprint match).
template <int W>
__device__ __forceinline__ long long lookup(const u64* q, u64 n_pre, const u64* keys, const u64* table, u64 mask,
                                            u64 bmask, SweepState* st) {
  const u64 h = key_hash<W>(q);
  const u32 fp = (u32)(h >> 32);
  const u64 b = bucket_start(h, mask, bmask);
  // slots b, b + 1 and the next two on the probe sequence (wrapping: a
  // bucket of 2 may be the table's last)
  const ulonglong2 s01 = __ldcg(reinterpret_cast<const ulonglong2*>(table + b));
  const ulonglong2 s23 = __ldcg(reinterpret_cast<const ulonglong2*>(table + ((b + 2) & mask)));
  const u64 sl[4] = {s01.x, s01.y, s23.x, s23.y};
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    if (sl[m] == EMPTY_SLOT) return -1;
    const u32 row = (u32)sl[m];
    if ((u32)(sl[m] >> 32) == fp && row < n_pre) {
      const u64* kp = keys + (u64)row * W;
      bool eq = true;
#pragma unroll
      for (int w = 0; w < W; ++w) eq &= __ldcg(kp + w) == q[w];
      if (eq) return row;
    }
  }
  return lookup_from<W>(q, fp, (b + 4) & mask, n_pre, keys, table, mask, st);
}

// lookup for a gate's partner search.  On a fingerprint match the candidate
// row's coefficient is loaded together with its key, so a found partner costs
// one round trip less (cj receives it); on a miss, `empty` receives the empty
// slot where the probe ended, which is the first slot an insert of q would
// take (every slot before it on q's probe sequence is occupied, and occupied
// slots stay occupied during an op), or NO_SLOT.  The coefficient is loaded
// only for candidate rows >= c_from (cj stays 0 below): a row that owns a
// pair only when its partner's index is higher passes its own index + 1 and
// saves, for every pair it does not own, a random sector it would not use.
template <int W>
__device__ long long lookup_from_c(const u64* q, u32 fp, u64 i, u64 n_pre, const u64* keys, const double* coeffs,
                                   const u64* table, u64 mask, SweepState* st, double& cj, u64& empty, u64 c_from) {
  for (u64 probe = 0; probe <= mask; ++probe) {
    const u64 s = __ldcg(table + i);
    if (s == EMPTY_SLOT) {
      empty = i;
      return -1;
    }
    const u32 row = (u32)s;
    if ((u32)(s >> 32) == fp && row < n_pre) {
      const u64* kp = keys + (u64)row * W;
      const double c = row >= c_from ? __ldcg(coeffs + row) : 0.0;
      bool eq = true;
#pragma unroll
      for (int w = 0; w < W; ++w) eq &= __ldcg(kp + w) == q[w];
      if (eq) {
        cj = c;
        return row;
      }
    }
    i = (i + 1) & mask;
  }
  atomicOr(&st->error, ERR_PROBE_OVERFLOW);
  empty = NO_SLOT;
  return -1;
}
template <int W>
__device__ __forceinline__ long long lookup_c(const u64* q, u64 n_pre, const u64* keys, const double* coeffs,
                                              const u64* table, u64 mask, u64 bmask, SweepState* st, double& cj,
                                              u64& empty, u64 c_from) {
  const u64 h = key_hash<W>(q);
  const u32 fp = (u32)(h >> 32);
  const u64 b = bucket_start(h, mask, bmask);
  // slots b, b + 1 and the next two on the probe sequence (wrapping: a
  // bucket of 2 may be the table's last)
  const ulonglong2 s01 = __ldcg(reinterpret_cast<const ulonglong2*>(table + b));
  const ulonglong2 s23 = __ldcg(reinterpret_cast<const ulonglong2*>(table + ((b + 2) & mask)));
  const u64 sl[4] = {s01.x, s01.y, s23.x, s23.y};
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    if (sl[m] == EMPTY_SLOT) {
      empty = (b + m) & mask;
      return -1;
    }
    const u32 row = (u32)sl[m];
    if ((u32)(sl[m] >> 32) == fp && row < n_pre) {
      const u64* kp = keys + (u64)row * W;
      const double c = row >= c_from ? __ldcg(coeffs + row) : 0.0;
      bool eq = true;
#pragma unroll
      for (int w = 0; w < W; ++w) eq &= __ldcg(kp + w) == q[w];
      if (eq) {
        cj = c;
        return row;
      }
    }
  }
  return lookup_from_c<W>(q, fp, (b + 4) & mask, n_pre, keys, coeffs, table, mask, st, cj, empty, c_from);
}

// Slot value v for q placed from `start`, the empty slot a lookup of q in
// this op ended on: the first attempt is the atomic itself, with no load
// before it; if another key took the slot meanwhile, the probe goes on as in
// insert.  Returns the slot, or NO_SLOT if the table is full.
template <int W>
__device__ u64 place_from(const u64* q, u64 v, u64 start, u64* table, u64 mask, u64 bmask, u32* error) {
  u64 i;
  if (start != NO_SLOT) {
    if (atomicCAS(table + start, EMPTY_SLOT, v) == EMPTY_SLOT) return start;
    i = (start + 1) & mask;
  } else {
    i = bucket_start(key_hash<W>(q), mask, bmask);
  }
  for (u64 probe = 0; probe <= mask; ++probe) {
    if (__ldcg(table + i) == EMPTY_SLOT && atomicCAS(table + i, EMPTY_SLOT, v) == EMPTY_SLOT) return i;
    i = (i + 1) & mask;
  }
  atomicOr(error, ERR_PROBE_OVERFLOW);
  return NO_SLOT;
}

// -(Im phase) of G*K = i^p * sign: the sin-branch multiplier (coeff.rs:151-168).
__device__ __forceinline__ double neg_im(int p, double sign) {
  return p == 1 ? -sign : (p == 3 ? sign : 0.0);
}

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

struct TileSmem {
  u32 tile;
  u32 excl;
  u32 cnt[32];  // item-major per-warp counts, then their exclusive prefixes
  u32 rec_on;   // adjoint recording of the running op (see SweepArgs::rec_idx)
  u64 rec_base, rec_key_base;
};

// Item-major block scan of IT flags per thread, then the look-back.  Leaves
// each (item, warp) exclusive rank base in sm.cnt and the tile's global
// exclusive prefix in sm.excl; the last tile publishes the op's new count.
template <int IT>
__device__ __forceinline__ void tile_scan(u32 flags, unsigned* masks, TileSmem& sm, u64* status, u32 t, u32 ntiles,
                                          u64 n_base, u32 epoch, SweepState* st, u64* n_out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < IT; ++k) {
    masks[k] = __ballot_sync(FULL, (flags >> k) & 1u);
    if (lane == 0) sm.cnt[k * NWARPS + warp] = __popc(masks[k]);
  }
  __syncthreads();
  if (warp == 0) {
    const u32 v = lane < IT * NWARPS ? sm.cnt[lane] : 0u;
    u32 inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 y = __shfl_up_sync(FULL, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane < IT * NWARPS) sm.cnt[lane] = inc - v;
    const u32 agg = __shfl_sync(FULL, inc, 31);
    const u32 excl = lookback(status, t, agg, epoch, st);
    if (lane == 0) {
      sm.excl = excl;
      if (t == ntiles - 1) st_volatile(n_out, n_base + excl + agg);
    }
  }
  __syncthreads();
}

// Adjoint recording of one gate's sin branches (see SweepArgs::rec_idx).  A
// source without a partner row records REC_NONE here; its child's row
// replaces it once the child is placed.
__device__ __forceinline__ void record_single(const SweepArgs& a, const TileSmem& sm, u64 r, double c) {
  const u64 o = sm.rec_base;
  a.rec_coef[o + r] = c;
  a.rec_idx[o + r] = REC_NONE;
}
__device__ __forceinline__ void record_pair(const SweepArgs& a, const TileSmem& sm, u64 r, u64 j, double c, double cj,
                                            bool to_j, bool to_i) {
  const u64 o = sm.rec_base;
  a.rec_coef[o + r] = c;
  a.rec_coef[o + j] = cj;
  a.rec_idx[o + r] = to_j ? (u32)j : REC_NONE;
  a.rec_idx[o + j] = to_i ? (u32)r : REC_NONE;
}

// Verbose-log accounting of one source row's sin branch (termsum.rs:604-751):
// a branch the emit check holds back counts as declined, and as discarded
// (|b| into the sum and the maximum) unless the partner claims it; a branch
// that goes out counts as emitted, and as a hit when it lands on an existing
// row.  |b| >= 0, so its bit pattern orders like the value for atomicMax.
__device__ __noinline__ void log_branch(u64* log, u32 op, int state, bool sent, bool hit, double b) {
  u64* l = log + (u64)op * LOG_WORDS;
  if (state == S_HELD) atomicAdd(l + LOG_HELD, 1ull);
  if (sent) {
    atomicAdd(l + LOG_EMITTED, 1ull);
    if (hit) atomicAdd(l + LOG_HITS, 1ull);
  } else if (state == S_HELD) {
    const double m = fabs(b);
    atomicAdd(reinterpret_cast<double*>(l + LOG_L1), m);
    atomicMax(l + LOG_MAX, (u64)__double_as_longlong(m));
  }
}

// ------------------------------------------------------------------ gate
// Tiles are assigned statically (tile t to block t mod grid, in order); the
// cooperative launch keeps every block resident, so a tile's look-back always
// waits on blocks that are running.
template <int W, int ALG, int IT>
__device__ __noinline__ void gate_tiles(const SweepArgs& a, const GateDesc<W>& d, u32 op, u64 N, u64* keys,
                                           double* coeffs, TileSmem& sm, const Grp grp, u64* n_out) {
  using Ops = typename Alg<ALG>::T;
  constexpr int TL = BLOCK * IT;
  SweepState* st = a.st;
  const u32 ntiles = (u32)((N + TL - 1) / TL);
  // TermBudget: below the floor every lossy predicate is off (termsum.rs:60-76).
  const bool lossless = a.min_terms && N < a.min_terms;
  const u32 wcut = lossless ? NO_WEIGHT_CUT : a.max_weight;
  const bool ccut = !lossless && a.has_min_coeff;
  const double minc = a.min_coeff;
  const double sn = d.sn, cs = d.cs;
  const GenInfo<W>& g = d.g;
  const u32 epoch = a.epoch_base + op;
  // Emit state of a source with coefficient c and child key ch
  // (termsum.rs:701-751): HELD by the magnitude precheck, DROP by weight, else EMIT.
  auto state = [&](double c, const u64* ch) -> int {
    if (ccut && fabs(__dmul_rn(c, sn)) < minc) return S_HELD;
    if (wcut != NO_WEIGHT_CUT && Ops::template weight<W>(ch, a.n_units) > wcut) return S_DROP;
    return S_EMIT;
  };
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u32 n_anti = 0;
  for (u32 t = grp.bid; t < ntiles; t += grp.nblk) {
    u64 key[IT][W];
    u32 anti = 0;
#pragma unroll
    for (int k = 0; k < IT; ++k) {
      const u64 r = (u64)t * TL + (u64)k * BLOCK + threadIdx.x;
      if (r < N) load_key<W>(keys, r, key[k]);
    }
#pragma unroll
    for (int k = 0; k < IT; ++k) {
      const u64 r = (u64)t * TL + (u64)k * BLOCK + threadIdx.x;
      if (r < N && Ops::template anticommutes<W>(g, key[k])) anti |= 1u << k;
    }
    n_anti += __popc(anti);
    // A row's own coefficient is loaded beside its partner lookup, and the
    // partner's coefficient inside it (lookup_c).
    long long j[IT];
    double c[IT], cj[IT];
    u64 es[IT];
#pragma unroll
    for (int k = 0; k < IT; ++k) {
      j[k] = -1;
      cj[k] = 0.0;
      es[k] = NO_SLOT;
      if (!((anti >> k) & 1u)) continue;
      const u64 r = (u64)t * TL + (u64)k * BLOCK + threadIdx.x;
      c[k] = __ldcg(coeffs + r);
      u64 q[W];
#pragma unroll
      for (int w = 0; w < W; ++w) q[w] = key[k][w] ^ g.gen[w];
      j[k] = lookup_c<W>(q, N, keys, coeffs, a.table, a.table_mask, a.table_bmask, st, cj[k], es[k], r + 1);
    }
    // The lower row of a pair owns both coefficients.
    u32 own = 0;
#pragma unroll
    for (int k = 0; k < IT; ++k) {
      const u64 r = (u64)t * TL + (u64)k * BLOCK + threadIdx.x;
      if (!((anti >> k) & 1u) || (j[k] >= 0 && (u64)j[k] < r)) continue;
      own |= 1u << k;
    }
    u32 emit = 0;
    double bval[IT];
    u64 slot[IT];
#pragma unroll
    for (int k = 0; k < IT; ++k) {
      bval[k] = 0.0;
      if (!((own >> k) & 1u)) continue;
      const u64 r = (u64)t * TL + (u64)k * BLOCK + threadIdx.x;
      u64 q[W];
#pragma unroll
      for (int w = 0; w < W; ++w) q[w] = key[k][w] ^ g.gen[w];
      const double bi = __dmul_rn(__dmul_rn(c[k], sn), neg_im(Ops::template product_exp<W>(g, key[k]), g.sign));
      const int si = a.host_state ? (int)a.host_state[r] : state(c[k], q);
      if (j[k] < 0) {
        coeffs[r] = __dmul_rn(c[k], cs);
        if (si == S_EMIT) {
          emit |= 1u << k;
          bval[k] = bi;
          slot[k] = place_from<W>(q, ((key_hash<W>(q) >> 32) << 32) | PENDING_ROW, es[k], a.table, a.table_mask, a.table_bmask,
                                  &st->error);
        }
        if (sm.rec_on) record_single(a, sm, r, c[k]);
        if (a.log) log_branch(a.log, op, si, si == S_EMIT, false, bi);
      } else {
        const double bj = __dmul_rn(__dmul_rn(cj[k], sn), neg_im(Ops::template product_exp<W>(g, q), g.sign));
        const int sj = a.host_state ? (int)a.host_state[j[k]] : state(cj[k], key[k]);
        const bool to_j = si == S_EMIT || (si == S_HELD && sj == S_EMIT);
        const bool to_i = sj == S_EMIT || (sj == S_HELD && si == S_EMIT);
        double ni = __dmul_rn(c[k], cs);
        if (to_i) ni = __dadd_rn(ni, bj);
        double nj = __dmul_rn(cj[k], cs);
        if (to_j) nj = __dadd_rn(nj, bi);
        coeffs[r] = ni;
        coeffs[j[k]] = nj;
        if (sm.rec_on) record_pair(a, sm, r, (u64)j[k], c[k], cj[k], to_j, to_i);
        if (a.log) {
          log_branch(a.log, op, si, to_j, true, bi);
          log_branch(a.log, op, sj, to_i, true, bj);
        }
      }
    }
    unsigned masks[IT];
    tile_scan<IT>(emit, masks, sm, a.status, t, ntiles, N, epoch, st, n_out);
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int k = 0; k < IT; ++k) {
      if (!((emit >> k) & 1u)) continue;
      const u64 row = N + sm.excl + sm.cnt[k * NWARPS + warp] + __popc(masks[k] & lt);
      if (row >= a.cap) {
        atomicOr(&st->error, ERR_CAPACITY);
        continue;
      }
      u64 q[W];
#pragma unroll
      for (int w = 0; w < W; ++w) q[w] = key[k][w] ^ g.gen[w];
      store_key<W>(keys, row, q);
      coeffs[row] = bval[k];
      set_row(a.table, slot[k], row);
      if (sm.rec_on) a.rec_idx[sm.rec_base + (u64)t * TL + (u64)k * BLOCK + threadIdx.x] = (u32)row;
    }
    __syncthreads();  // sm is reused by the next tile
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) n_anti += __shfl_xor_sync(FULL, n_anti, o);
  if (lane == 0 && n_anti && a.anti) atomicAdd(a.anti + op, (u64)n_anti);
}

// Many rows: tiles of `its` x BLOCK rows (its = SweepArgs::tile_items, 1 to
// MAX_ITEMS) handed out in order by a per-op ticket, each thread taking its
// rows one after the other.
template <int W, int ALG>
__device__ __noinline__ void gate_tiles_large(const SweepArgs& a, const GateDesc<W>& d, u32 op, u64 N, u64* keys,
                                                 double* coeffs, TileSmem& sm, u64* n_out) {
  using Ops = typename Alg<ALG>::T;
  constexpr int IT = MAX_ITEMS;
  const u32 its = a.tile_items && a.tile_items < (u32)IT ? a.tile_items : (u32)IT;
  const u64 TL = (u64)BLOCK * its;
  SweepState* st = a.st;
  const u32 ntiles = (u32)((N + TL - 1) / TL);
  const bool lossless = a.min_terms && N < a.min_terms;
  const u32 wcut = lossless ? NO_WEIGHT_CUT : a.max_weight;
  const bool ccut = !lossless && a.has_min_coeff;
  const double minc = a.min_coeff;
  const double sn = d.sn, cs = d.cs;
  const GenInfo<W>& g = d.g;
  const u32 epoch = a.epoch_base + op;
  auto state = [&](double c, const u64* ch) -> int {
    if (ccut && fabs(__dmul_rn(c, sn)) < minc) return S_HELD;
    if (wcut != NO_WEIGHT_CUT && Ops::template weight<W>(ch, a.n_units) > wcut) return S_DROP;
    return S_EMIT;
  };
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u32 n_anti = 0;
  for (;;) {
    if (threadIdx.x == 0) sm.tile = atomicAdd(a.tickets + op, 1u);
    __syncthreads();
    const u32 t = sm.tile;
    if (t >= ntiles) break;
    u32 emit = 0;
    double bval[IT];
    u64 eslot[IT];
#pragma unroll
    for (int k = 0; k < IT; ++k) {
      bval[k] = 0.0;
      const u64 r = (u64)t * TL + (u64)k * BLOCK + threadIdx.x;
      if ((u32)k >= its || r >= N) continue;
      u64 key[W];
      load_key<W>(keys, r, key);
      if (!Ops::template anticommutes<W>(g, key)) continue;
      ++n_anti;
      const double c = __ldcg(coeffs + r);  // beside the lookup, not after it
      u64 q[W];
#pragma unroll
      for (int w = 0; w < W; ++w) q[w] = key[w] ^ g.gen[w];
      double cj = 0.0;
      u64 es = NO_SLOT;
      const long long j = lookup_c<W>(q, N, keys, coeffs, a.table, a.table_mask, a.table_bmask, st, cj, es, r + 1);
      if (j >= 0 && (u64)j < r) continue;  // the lower row of the pair owns it
      const double bi = __dmul_rn(__dmul_rn(c, sn), neg_im(Ops::template product_exp<W>(g, key), g.sign));
      const int si = a.host_state ? (int)a.host_state[r] : state(c, q);
      if (j < 0) {
        coeffs[r] = __dmul_rn(c, cs);
        if (si == S_EMIT) {
          emit |= 1u << k;
          bval[k] = bi;
          eslot[k] = es;
        }
        if (sm.rec_on) record_single(a, sm, r, c);
        if (a.log) log_branch(a.log, op, si, si == S_EMIT, false, bi);
      } else {
        const double bj = __dmul_rn(__dmul_rn(cj, sn), neg_im(Ops::template product_exp<W>(g, q), g.sign));
        const int sj = a.host_state ? (int)a.host_state[j] : state(cj, key);
        const bool to_j = si == S_EMIT || (si == S_HELD && sj == S_EMIT);
        const bool to_i = sj == S_EMIT || (sj == S_HELD && si == S_EMIT);
        double ni = __dmul_rn(c, cs);
        if (to_i) ni = __dadd_rn(ni, bj);
        double nj = __dmul_rn(cj, cs);
        if (to_j) nj = __dadd_rn(nj, bi);
        coeffs[r] = ni;
        coeffs[j] = nj;
        if (sm.rec_on) record_pair(a, sm, r, (u64)j, c, cj, to_j, to_i);
        if (a.log) {
          log_branch(a.log, op, si, to_j, true, bi);
          log_branch(a.log, op, sj, to_i, true, bj);
        }
      }
    }
    unsigned masks[IT];
    tile_scan<IT>(emit, masks, sm, a.status, t, ntiles, N, epoch, st, n_out);
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int k = 0; k < IT; ++k) {
      if (!((emit >> k) & 1u)) continue;
      const u64 r = (u64)t * TL + (u64)k * BLOCK + threadIdx.x;
      const u64 row = N + sm.excl + sm.cnt[k * NWARPS + warp] + __popc(masks[k] & lt);
      if (row >= a.cap) {
        atomicOr(&st->error, ERR_CAPACITY);
        continue;
      }
      u64 q[W];
      load_key<W>(keys, r, q);
#pragma unroll
      for (int w = 0; w < W; ++w) q[w] ^= g.gen[w];
      store_key<W>(keys, row, q);
      coeffs[row] = bval[k];
      place_from<W>(q, ((key_hash<W>(q) >> 32) << 32) | (row & 0xffffffffULL), eslot[k], a.table, a.table_mask, a.table_bmask,
                    &st->error);
      if (sm.rec_on) a.rec_idx[sm.rec_base + r] = (u32)row;
    }
    __syncthreads();
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) n_anti += __shfl_xor_sync(FULL, n_anti, o);
  if (lane == 0 && n_anti && a.anti) atomicAdd(a.anti + op, (u64)n_anti);
}

template <int W, int ALG>
__device__ __forceinline__ void gate_op(const SweepArgs& a, const GateDesc<W>& d, u32 op, u64 N, u64* keys,
                                        double* coeffs, TileSmem& sm, const Grp grp, u64* n_out) {
  if (N == 0) {
    if (grp.bid == 0 && threadIdx.x == 0) st_volatile(n_out, 0);
    return;
  }
  // Few rows: one row per thread and at most one 256-row tile per block, so
  // every row's chain of dependent loads runs at once.
  if (N <= (u64)grp.nblk * BLOCK)
    gate_tiles<W, ALG, 1>(a, d, op, N, keys, coeffs, sm, grp, n_out);
  else
    gate_tiles_large<W, ALG>(a, d, op, N, keys, coeffs, sm, n_out);
}

// Two rotations G1 then G2 whose generators commute, in one pass over the
// rows.  Since G1 G2 = G2 G1, the keys {K, K^G1, K^G2, K^G1^G2} (a family)
// all anticommute with G1 iff K does and with G2 iff K does, and no rotation
// moves a term out of its family; so the two sequential steps of the
// reference -- the pair rule for G1 on (K, K^G1) and (K^G2, K^G1^G2), then
// for G2 on (K, K^G2) and (K^G1, K^G1^G2) with the results -- can be run for
// each family by one thread: the present row of lowest index owns the family
// (rows look up the other members among the rows entering the op), writes the
// coefficients of its present members and appends the members that either
// step creates, with their final coefficients.  Every coefficient is the same
// two-operand result as in two separate passes; only the order in which the
// new rows are appended differs (deterministic: by owner row, then member).
// Not used with a TermBudget floor (its lossless switch reads the live count
// between the two rotations) or when recording for the adjoint.  The sweep
// runs it when every block has at most one tile (the latency-bound regime it
// is for); with more rows it runs the two rotations one after the other.
template <int W, int ALG>
__device__ __noinline__ void gate2_tiles(const SweepArgs& a, const GateDesc<W>& d1, const GateDesc<W>& d2, u32 op,
                                         u64 N, u64* keys, double* coeffs, TileSmem& sm, const Grp grp, u64* n_out) {
  using Ops = typename Alg<ALG>::T;
  constexpr int TL = BLOCK;
  SweepState* st = a.st;
  const u32 ntiles = (u32)((N + TL - 1) / TL);
  const u32 wcut = a.max_weight;
  const bool ccut = a.has_min_coeff != 0;
  const double minc = a.min_coeff;
  const u32 epoch = a.epoch_base + op;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u32 n_anti1 = 0, n_anti2 = 0, n_born1 = 0;
  for (u32 t = grp.bid; t < ntiles; t += grp.nblk) {
    const u64 r = (u64)t * TL + threadIdx.x;
    u64 k0[W];
    bool a1 = false, a2 = false;
    if (r < N) {
      load_key<W>(keys, r, k0);
      a1 = Ops::template anticommutes<W>(d1.g, k0);
      a2 = Ops::template anticommutes<W>(d2.g, k0);
    }
    n_anti1 += a1;
    n_anti2 += a2;
    // key of member m (bit 0: times G1, bit 1: times G2)
    auto member = [&](int m, u64* out) {
#pragma unroll
      for (int w = 0; w < W; ++w) out[w] = k0[w] ^ ((m & 1) ? d1.g.gen[w] : 0ull) ^ ((m & 2) ? d2.g.gen[w] : 0ull);
    };
    // The row's own coefficient is loaded beside the member lookups, the
    // members' coefficients inside them (lookup_c), and each lookup's miss
    // slot is where that member would be placed.
    long long j[4] = {(long long)r, -1, -1, -1};
    double cm[4] = {0.0, 0.0, 0.0, 0.0};
    u64 es[4] = {NO_SLOT, NO_SLOT, NO_SLOT, NO_SLOT};
    if (a1 || a2) cm[0] = __ldcg(coeffs + r);
    {
      u64 q[W];
      if (a1) {
        member(1, q);
        j[1] = lookup_c<W>(q, N, keys, coeffs, a.table, a.table_mask, a.table_bmask, st, cm[1], es[1], r + 1);
      }
      if (a2) {
        member(2, q);
        j[2] = lookup_c<W>(q, N, keys, coeffs, a.table, a.table_mask, a.table_bmask, st, cm[2], es[2], r + 1);
      }
      if (a1 && a2) {
        member(3, q);
        j[3] = lookup_c<W>(q, N, keys, coeffs, a.table, a.table_mask, a.table_bmask, st, cm[3], es[3], r + 1);
      }
    }
    const bool own = (a1 || a2) && (j[1] < 0 || (u64)j[1] > r) && (j[2] < 0 || (u64)j[2] > r) &&
                     (j[3] < 0 || (u64)j[3] > r);
    u32 emit = 0;
    double bval[3] = {0.0, 0.0, 0.0};
    u64 slot[3] = {NO_SLOT, NO_SLOT, NO_SLOT};
    if (own) {
      double c[4];
      bool p[4];
      int born[4] = {0, 0, 0, 0};  // the step that created the member (1 or 2), 0 if it entered the op
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        p[m] = j[m] >= 0;
        c[m] = p[m] ? cm[m] : 0.0;
      }
      // One reference step on the pair (x, y) of the family
      // (termsum.rs:604-751): the pair rule if both are present, else the
      // lone member's cos update and, on EMIT, the other member's creation.
      auto step = [&](const GateDesc<W>& d, int x, int y, int s) {
        if (!p[x] && !p[y]) return;
        u64 kx[W], ky[W];
        member(x, kx);
        member(y, ky);
        auto state = [&](double cv, const u64* ch) -> int {
          if (ccut && fabs(__dmul_rn(cv, d.sn)) < minc) return S_HELD;
          if (wcut != NO_WEIGHT_CUT && Ops::template weight<W>(ch, a.n_units) > wcut) return S_DROP;
          return S_EMIT;
        };
        if (p[x] && p[y]) {
          const double bx = __dmul_rn(__dmul_rn(c[x], d.sn), neg_im(Ops::template product_exp<W>(d.g, kx), d.g.sign));
          const double by = __dmul_rn(__dmul_rn(c[y], d.sn), neg_im(Ops::template product_exp<W>(d.g, ky), d.g.sign));
          const int sx = state(c[x], ky), sy = state(c[y], kx);
          const bool to_y = sx == S_EMIT || (sx == S_HELD && sy == S_EMIT);
          const bool to_x = sy == S_EMIT || (sy == S_HELD && sx == S_EMIT);
          double nx = __dmul_rn(c[x], d.cs);
          if (to_x) nx = __dadd_rn(nx, by);
          double ny = __dmul_rn(c[y], d.cs);
          if (to_y) ny = __dadd_rn(ny, bx);
          c[x] = nx;
          c[y] = ny;
        } else {
          const int l = p[x] ? x : y, o = p[x] ? y : x;
          const u64* kl = p[x] ? kx : ky;
          const u64* ko = p[x] ? ky : kx;
          const double b = __dmul_rn(__dmul_rn(c[l], d.sn), neg_im(Ops::template product_exp<W>(d.g, kl), d.g.sign));
          const int sl = state(c[l], ko);
          c[l] = __dmul_rn(c[l], d.cs);
          if (sl == S_EMIT) {
            p[o] = true;
            c[o] = b;
            born[o] = s;
          }
        }
      };
      if (a1) {
        step(d1, 0, 1, 1);
        if (a2) step(d1, 2, 3, 1);
      }
      if (a2) {
        step(d2, 0, 2, 2);
        if (a1) step(d2, 1, 3, 2);
      }
#pragma unroll
      for (int m = 0; m < 4; ++m)
        if (j[m] >= 0) coeffs[j[m]] = c[m];
#pragma unroll
      for (int m = 1; m < 4; ++m) {
        if (!born[m]) continue;
        emit |= 1u << (m - 1);
        bval[m - 1] = c[m];
        u64 q[W];
        member(m, q);
        // before the scan: see claim_slot
        slot[m - 1] = place_from<W>(q, ((key_hash<W>(q) >> 32) << 32) | PENDING_ROW, es[m], a.table, a.table_mask, a.table_bmask,
                                    &st->error);
        if (born[m] == 1) {
          ++n_born1;
          if (a2) ++n_anti2;  // a row the first rotation creates here anticommutes with the second
        }
      }
    }
    unsigned masks[3];
    tile_scan<3>(emit, masks, sm, a.status, t, ntiles, N, epoch, st, n_out);
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (!((emit >> k) & 1u)) continue;
      const u64 row = N + sm.excl + sm.cnt[k * NWARPS + warp] + __popc(masks[k] & lt);
      if (row >= a.cap) {
        atomicOr(&st->error, ERR_CAPACITY);
        continue;
      }
      u64 q[W];
      member(k + 1, q);
      store_key<W>(keys, row, q);
      coeffs[row] = bval[k];
      set_row(a.table, slot[k], row);
    }
    __syncthreads();  // sm is reused by the next tile
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    n_anti1 += __shfl_xor_sync(FULL, n_anti1, o);
    n_anti2 += __shfl_xor_sync(FULL, n_anti2, o);
    n_born1 += __shfl_xor_sync(FULL, n_born1, o);
  }
  if (lane == 0) {
    if (n_anti1 && a.anti) atomicAdd(a.anti + op, (u64)n_anti1);
    if (n_anti2 && a.anti) atomicAdd(a.anti + op + 1, (u64)n_anti2);
    if (n_born1) atomicAdd(a.tickets + op, n_born1);  // rows after the first rotation: N + this
  }
}

// A rotation with |sin| < 1e-9 only scales the anticommuting rows by cos
// (partitioned_termsum.rs:303-308, termsum.rs:551-557).
template <int W, int ALG>
__device__ __noinline__ void phase_op(const SweepArgs& a, const GateDesc<W>& d, u32 op, u64 N, const u64* keys,
                                      double* coeffs, const TileSmem& sm, const Grp grp) {
  using Ops = typename Alg<ALG>::T;
  for (u64 r = (u64)grp.bid * BLOCK + threadIdx.x; r < N; r += (u64)grp.nblk * BLOCK) {
    u64 key[W];
    load_key<W>(keys, r, key);
    if (Ops::template anticommutes<W>(d.g, key)) {
      const double c = __ldcg(coeffs + r);
      coeffs[r] = __dmul_rn(c, d.cs);
      if (sm.rec_on) a.rec_coef[sm.rec_base + r] = c;
    }
  }
}

// Noise without truncation: c *= factor[min(w, len-1)] (engine.rs:119-125).
template <int W, int ALG>
__device__ __noinline__ void noise_scale_op(const SweepArgs& a, const double* factors, u64 N, const u64* keys,
                                               double* coeffs, const Grp grp) {
  using Ops = typename Alg<ALG>::T;
  const u32 last = a.table_len - 1;
  for (u64 r = (u64)grp.bid * BLOCK + threadIdx.x; r < N; r += (u64)grp.nblk * BLOCK) {
    u64 key[W];
    load_key<W>(keys, r, key);
    const u32 w = Ops::template weight<W>(key, a.n_units);
    const double f = a.host_factor ? __ldg(a.host_factor + r) : __ldg(factors + (w < last ? w : last));
    coeffs[r] = __dmul_rn(__ldcg(coeffs + r), f);
  }
}

// Noise with truncation: damp, keep weight <= cut and |c| >= cut
// (partitioned_termsum.rs:581-608), compact survivors in row order into the
// other buffer and re-insert them into the cleared table.
template <int W, int ALG>
__device__ __noinline__ void noise_compact_op(const SweepArgs& a, const double* factors, u32 op, u64 N,
                                                 const u64* keys, const double* coeffs, u64* keys_out,
                                                 double* coeffs_out, TileSmem& sm, const Grp grp, u64* n_out) {
  using Ops = typename Alg<ALG>::T;
  constexpr int IT = 1;
  constexpr int TL = BLOCK * IT;
  SweepState* st = a.st;
  const u32 ntiles = (u32)((N + TL - 1) / TL);
  if (ntiles == 0) {
    if (grp.bid == 0 && threadIdx.x == 0) st_volatile(n_out, 0);
    return;
  }
  const u32 last = a.table_len - 1;
  const u32 epoch = a.epoch_base + op;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (u32 t = grp.bid; t < ntiles; t += grp.nblk) {
    u32 keep = 0;
    double cv[IT];
    u64 key[IT][W];
    u64 slot[IT];
#pragma unroll
    for (int k = 0; k < IT; ++k) {
      const u64 r = (u64)t * TL + (u64)k * BLOCK + threadIdx.x;
      if (r < N) {
        load_key<W>(keys, r, key[k]);
        cv[k] = __ldcg(coeffs + r);
      }
    }
#pragma unroll
    for (int k = 0; k < IT; ++k) {
      const u64 r = (u64)t * TL + (u64)k * BLOCK + threadIdx.x;
      if (r >= N) continue;
      const u32 w = Ops::template weight<W>(key[k], a.n_units);
      const double f = a.host_factor ? __ldg(a.host_factor + r) : __ldg(factors + (w < last ? w : last));
      const double c = __dmul_rn(cv[k], f);
      cv[k] = c;
      const bool kp = a.host_keep ? a.host_keep[r] != 0
                                  : (a.max_weight == NO_WEIGHT_CUT || w <= a.max_weight) &&
                                        (!a.has_min_coeff || fabs(c) >= a.min_coeff);
      keep |= (u32)kp << k;
      if (kp) slot[k] = claim_slot<W>(key[k], a.table, a.table_mask, a.table_bmask, &st->error);
      if (sm.rec_on) {
        a.rec_idx[sm.rec_base + r] = REC_NONE;
        store_key<W>(a.rec_keys + sm.rec_key_base * W, r, key[k]);
      }
    }
    unsigned masks[IT];
    tile_scan<IT>(keep, masks, sm, a.status, t, ntiles, 0, epoch, st, n_out);
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int k = 0; k < IT; ++k) {
      if (!((keep >> k) & 1u)) continue;
      const u64 row = sm.excl + sm.cnt[k * NWARPS + warp] + __popc(masks[k] & lt);
      store_key<W>(keys_out, row, key[k]);
      coeffs_out[row] = cv[k];
      set_row(a.table, slot[k], row);
      if (sm.rec_on) a.rec_idx[sm.rec_base + (u64)t * TL + (u64)k * BLOCK + threadIdx.x] = (u32)row;
    }
    __syncthreads();
  }
}

#include "pq_class.cuh"

// Runs ops [a.op_begin, a.op_end) of one propagation on the blocks of `grp`.
// 8-byte asynchronous copy global -> shared (cp.async; completes at cp_async_wait).
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  const u32 d = (u32)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <int W, int ALG>
__device__ __forceinline__ void sweep_body(const SweepArgs& a, const Grp grp) {
  __shared__ TileSmem sm;
  // The running op's descriptor and generator(s) in buffer sb; the next op's
  // are copied into the other buffer while the running op works.
  __shared__ __align__(16) GateDesc<W> sgs[2][4];
  __shared__ __align__(8) OpDesc sod[2];
  __shared__ OpShared os;
  SweepState* st = a.st;
  u32 gen = *(volatile u32*)&st->bar_gen;
  int cur = (int)a.cur0;
  u32 op = a.op_begin;
  u32 sb = 0;
  // The live count entering the next op is in n[par]; each op writes
  // n[par ^ 1].  (Not n[op & 1]: a fused op is several ops.)
  u32 par = op & 1u;
  const GateDesc<W>* gdesc = reinterpret_cast<const GateDesc<W>*>(a.gates);
  auto rotation_op = [](u32 kind) {
    return kind != OP_NOISE_SCALE && kind != OP_NOISE_COMPACT && !is_class(kind);
  };
  // Thread 0: op k's descriptors into buffer b, synchronously.
  auto fetch_op = [&](u32 k, u32 b) {
    if (k >= a.op_end) return;
    const OpDesc d = a.ops[k];
    sod[b] = d;
    if (rotation_op(d.kind))
      for (u32 i = 0; i < fused_count(d.kind); ++i) sgs[b][i] = gdesc[d.idx + i];
  };
  // Warp 0, at the start of an op: the copies of op k's descriptor and of the
  // gate descriptors from gi on (those of the next rotation op -- gate
  // descriptors are in op order) into buffer b.  Returns how many gate
  // descriptors it copies.
  auto prefetch_op = [&](u32 k, u32 gi, u32 b) -> u32 {
    if (k >= a.op_end) return 0;
    const u32 lane = threadIdx.x & 31;
    if (lane == 0) cp_async8(&sod[b], a.ops + k);
    const u32 ng = gi < a.n_gdesc ? (a.n_gdesc - gi < 4u ? a.n_gdesc - gi : 4u) : 0u;
    constexpr u32 WORDS = sizeof(GateDesc<W>) / 8;
    static_assert(sizeof(GateDesc<W>) % 8 == 0, "gate descriptors copy in 8-byte words");
    const u64* src = reinterpret_cast<const u64*>(gdesc + gi);
    u64* dst = reinterpret_cast<u64*>(&sgs[b][0]);
    for (u32 w = lane; w < ng * WORDS; w += 32) cp_async8(dst + w, src + w);
    return ng;
  };
  if (threadIdx.x == 0) {
    fetch_op(op, 0);
    os.n = ld_volatile(&st->n[par]);
    sm.rec_on = 0;
  }
  u32 g_next = 0;  // warp 0: the gate descriptor the next rotation op is expected to start at
  // Block 0, thread 0: the largest live count this launch has seen.
  u64 peak = (grp.bid == 0 && threadIdx.x == 0) ? ld_volatile(&st->peak) : 0;
  // Adjoint recording: every block places the ops identically from the same
  // live counts, so the offsets agree without communication.
  u64 rb = a.rec_idx ? ld_volatile(&st->rec_next) : 0, rkb = a.rec_idx ? ld_volatile(&st->rec_key_next) : 0;
  bool rec_on = a.rec_idx && !*(volatile u32*)&st->rec_full;
  if (a.hold_us && grp.bid == a.hold_block && threadIdx.x == 0) {
    // failure tests only: a bounded hold, so the others' waits on this block expire
    u64 t0, t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (u32 i = 0; i < (1u << 20); ++i) {  // the host caps hold_us at 100 ms
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      if (t - t0 >= (u64)a.hold_us * 1000ull) break;
      __nanosleep(1000);
    }
  }
  __syncthreads();
  bool stopped = false;  // a capacity stop inside a fused op
  while (op < a.op_end) {
    OpDesc od = sod[sb];
    const GateDesc<W>* sg = sgs[sb];
    // A launch that resumes inside a fused group (after a capacity stop) runs
    // the remaining rotations as plain ones.
    if (od.kind == OP_GATE_TAIL) od.kind = OP_GATE;
    const u64 N = os.n;
    u64* keys = a.keys[cur];
    double* coeffs = a.coeffs[cur];
    u64* n_out = &st->n[par ^ 1u];
    const u32 nops = fused_count(od.kind);
    bool split = false;  // a fused op that ran its rotations one after the other
    const bool gate_like = od.kind != OP_NOISE_SCALE && od.kind != OP_NOISE_COMPACT;
    if (gate_like && 2 * N > a.cap) {  // uniform: every block reads the same N
      if (grp.bid == 0 && threadIdx.x == 0) st->halt = op;
      break;
    }
    if (a.grid_rows && N > a.grid_rows) {  // the host relaunches on a larger grid
      if (grp.bid == 0 && threadIdx.x == 0) {
        st->halt = op;
        st->grid_stop = 1;
      }
      break;
    }
    // The next op's descriptors, copied while this one runs: gate descriptors
    // follow this op's (or stay where they were after a noise op).
    u32 g_pred = 0, g_copied = 0;
    if (threadIdx.x < 32) {
      if (rotation_op(od.kind) || is_class(od.kind)) g_next = od.idx + nops;
      g_pred = g_next;
      g_copied = prefetch_op(op + nops, g_pred, sb ^ 1u);
    }
    if (a.rec_idx) {
      const bool rec_op = gate_like || od.kind == OP_NOISE_COMPACT;
      if (rec_on && rec_op &&
          (rb + N > a.rec_cap || (od.kind == OP_NOISE_COMPACT && rkb + N > a.rec_key_cap)))
        rec_on = false;  // the pool is full: this op and every later one go unrecorded
      if (threadIdx.x == 0) {
        sm.rec_on = rec_on && rec_op;
        sm.rec_base = rb;
        sm.rec_key_base = rkb;
        if (grp.bid == 0) {
          a.rec_off[op] = rb;
          a.rec_key_off[op] = rkb;
        }
      }
      __syncthreads();
      if (rec_on && rec_op) {
        rb += N;
        if (od.kind == OP_NOISE_COMPACT) rkb += N;
      }
    }
    if (gate_like) {
      if (od.kind == OP_GATE) {
        gate_op<W, ALG>(a, sg[0], op, N, keys, coeffs, sm, grp, n_out);
      } else if (od.kind == OP_PHASE) {
        phase_op<W, ALG>(a, sg[0], op, N, keys, coeffs, sm, grp);
        if (grp.bid == 0 && threadIdx.x == 0) st_volatile(n_out, N);
      } else if (N == 0) {
        if (grp.bid == 0 && threadIdx.x == 0) st_volatile(n_out, 0);
      } else if (is_class(od.kind)) {
        const GateDesc<W>* gd = reinterpret_cast<const GateDesc<W>*>(a.gates) + od.idx;
        int rc = 1;
        if constexpr (W <= 4)
          rc = class_op<W, ALG>(a, gd, nops, op, N, keys, coeffs, sm, grp, n_out, gen);
        else if (threadIdx.x == 0)  // the host forms classes for keys of at most 4 words
          atomicOr(&st->error, ERR_CLASS_FAMILY);
        if (rc == 2) {  // capacity: stopped before any write, st->halt is set
          stopped = true;
          break;
        }
        // rc 1: a device error; the barrier below ends the sweep
      } else if (nops == 2 && N <= (u64)grp.nblk * BLOCK * GATE2_TILES_PER_BLOCK && 4 * N <= a.cap) {
        gate2_tiles<W, ALG>(a, sg[0], sg[1], op, N, keys, coeffs, sm, grp, n_out);
      } else {  // many rows: the rotations one after the other (op + i is rotation i's slot)
        split = true;
        u64 Ni = N;
        for (u32 i = 0; i < nops; ++i) {
          if (i > 0 && 2 * Ni > a.cap) {  // stop before rotation i
            if (grp.bid == 0 && threadIdx.x == 0) {
              st->n[par] = Ni;  // read as the next op's count (nobody reads n[par] during this op)
              st->halt = op + i;
              if (Ni > peak) peak = Ni;
            }
            op += i;
            stopped = true;
            break;
          }
          u64* out_i = i + 1 == nops ? n_out : &st->n_mid[i & 1];
          gate_op<W, ALG>(a, sg[i], op + i, Ni, keys, coeffs, sm, grp, out_i);
          if (i + 1 < nops) {
            grid_barrier(st, gen, grp);
            Ni = ld_volatile(out_i);
            if (grp.bid == 0 && threadIdx.x == 0) {
              a.hist[op + i] = Ni;
              if (a.stamps) {  // a capacity stop before the next rotation leaves no other stamp for this one
                u64 t;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                a.stamps[op + i] = t;
              }
            }
          }
        }
        if (stopped) break;
      }
    } else if (od.kind == OP_NOISE_SCALE) {
      noise_scale_op<W, ALG>(a, a.tables + (u64)od.idx * a.table_len, N, keys, coeffs, grp);
      if (grp.bid == 0 && threadIdx.x == 0) st_volatile(n_out, N);
    } else {
      for (u64 i = (u64)grp.bid * BLOCK + threadIdx.x; i <= a.table_mask; i += (u64)grp.nblk * BLOCK)
        a.table[i] = EMPTY_SLOT;
      grid_barrier(st, gen, grp);
      noise_compact_op<W, ALG>(a, a.tables + (u64)od.idx * a.table_len, op, N, keys, coeffs, a.keys[cur ^ 1],
                               a.coeffs[cur ^ 1], sm, grp, n_out);
      cur ^= 1;
    }
    // In a batch, once enough of the grid sits idle every instance stops at
    // this op boundary so that the host can hand the idle blocks to the
    // instances still running.  Block 0 names the op before the barrier and
    // every block compares it with its own op after it, so all blocks take
    // the same branch (a block reading late sees a later op and goes on).
    if (a.idle_blocks && grp.bid == 0 && threadIdx.x == 0 && *(volatile u32*)a.idle_blocks >= a.yield_at)
      *(volatile u32*)&st->yield_after = op + 1;
    const bool cls = is_class(od.kind) && !split;
    if (threadIdx.x < 32) cp_async_wait();  // the next op's descriptors, before the barrier's __syncthreads
    // After the release, thread 0 checks the copied descriptor: a rotation op
    // whose gate descriptors are not the ones copied is fetched again.
    op_barrier(st, gen, grp, n_out, nops > 1 && !split && !cls ? a.tickets + op : nullptr, nops - 1, os, [&] {
      const u32 k = op + nops;
      if (k >= a.op_end) return;
      const OpDesc d = sod[sb ^ 1u];
      if (rotation_op(d.kind) && (d.idx != g_pred || fused_count(d.kind) > g_copied)) fetch_op(k, sb ^ 1u);
    });
    par ^= 1u;
    if (os.err) {
      op += nops;
      break;
    }
    if (grp.bid == 0 && cls && threadIdx.x < 32) {
      // Counts after each rotation of the class but the last: the rows each
      // one created (tickets), summed over the class by a warp scan.
      u64 acc = N;
      for (u32 i0 = 0; i0 + 1 < nops; i0 += 32) {
        const u32 i = i0 + threadIdx.x;
        const u64 v = i + 1 < nops ? (u64)__ldcg(a.tickets + op + i) : 0ull;
        u64 inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const u64 y = __shfl_up_sync(FULL, inc, o);
          if ((int)threadIdx.x >= o) inc += y;
        }
        if (i + 1 < nops) a.hist[op + i] = acc + inc;
        acc += __shfl_sync(FULL, inc, 31);
      }
    }
    if (grp.bid == 0 && threadIdx.x == 0) {
      const u64 n_new = os.n;
      a.hist[op + nops - 1] = n_new;
      if (nops > 1 && !split && !cls) {  // counts after each rotation of the group but the last
        u64 acc = N;
        for (u32 i = 0; i + 1 < nops; ++i) {
          acc += os.extra[i];
          a.hist[op + i] = acc;
        }
      }
      if (n_new > peak) peak = n_new;
      if (a.stamps) {
        u64 t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        for (u32 i = 0; i < nops; ++i) a.stamps[op + i] = t;
      }
    }
    const bool stop = a.idle_blocks && os.yield_after == op + 1;
    op += nops;
    sb ^= 1u;
    if (stop) break;
  }
  if (threadIdx.x < 32) cp_async_wait();  // copies of an op the sweep stopped before
  if (grp.bid == 0 && threadIdx.x == 0) {
    if (peak > st->peak) st->peak = peak;
    st->cur = (u32)cur;
    st->end_op = op;
    if (a.rec_idx) {
      st->rec_next = rb;
      st->rec_key_next = rkb;
      st->rec_full = rec_on ? 0u : 1u;
    }
    // The host reads the live count at n[end_op & 1].
    if ((op & 1u) != par) st->n[op & 1u] = ld_volatile(&st->n[par]);
    if (a.idle_blocks) atomicAdd(a.idle_blocks, grp.nblk);
  }
}

template <int W>
struct MinBlocks {
  static constexpr int value = W >= 8 ? 2 : (W == 4 ? 3 : 4);
};

template <int W, int ALG>
__global__ void __launch_bounds__(BLOCK, MinBlocks<W>::value) sweep_kernel(const SweepArgs a) {
  sweep_body<W, ALG>(a, Grp{blockIdx.x, gridDim.x});
}

// The same sweep for 1- and 2-word keys, compiled for six resident blocks of
// 256 per SM (42 registers a thread) instead of four.  For live sets of
// 2^24 rows and more, where each op streams the rows from HBM, the extra
// warps in flight hide more of the random partner lookups (the 32-site
// Majorana run: 602 -> 562 ms); with fewer rows the registers of
// sweep_kernel win (the TFIM chain ran 11% slower at six blocks).
template <int W, int ALG>
__global__ void __launch_bounds__(BLOCK, 6) sweep_kernel_occ(const SweepArgs a) {
  sweep_body<W, ALG>(a, Grp{blockIdx.x, gridDim.x});
}

// The same sweep for keys of at most 4 words, compiled for two resident
// blocks of 256 per SM (up to 128 registers a thread, no spills in the op
// paths): the grids of one and two blocks per SM that small and mid-size live
// sets run on.
template <int W, int ALG>
__global__ void __launch_bounds__(BLOCK, 2) sweep_kernel_two(const SweepArgs a) {
  sweep_body<W, ALG>(a, Grp{blockIdx.x, gridDim.x});
}

// A batch: each instance owns the contiguous blocks [blk_begin, blk_begin +
// blk_count) of the cooperative grid and runs its own op sequence with its own
// barrier; block_inst maps a block to its instance.  Instances run at WM or
// WM / 2 words, so one launch holds, e.g., 64-unit and 128-unit registers.
// The batch kernel holds instances at WM and WM / 2 words; with WM = 4 it
// runs best at four resident blocks per SM (64 registers): the 64-instance
// sweep took 980 ms against 1,031 ms at three.
template <int WM>
struct BatchMinBlocks {
  static constexpr int value = WM == 4 ? 4 : MinBlocks<WM>::value;
};

template <int WM, int ALG>
__global__ void __launch_bounds__(BLOCK, BatchMinBlocks<WM>::value) batch_sweep_kernel(const SweepArgs* args,
                                                                                const u32* block_inst) {
  __shared__ SweepArgs sa;
  if (threadIdx.x == 0) sa = args[block_inst[blockIdx.x]];
  __syncthreads();
  const Grp grp{blockIdx.x - sa.blk_begin, sa.blk_count};
  if constexpr (WM > 1) {
    if (sa.n_words != WM) {
      sweep_body<WM / 2, ALG>(sa, grp);
      return;
    }
  }
  sweep_body<WM, ALG>(sa, grp);
}

// ------------------------------------------------------------ expectation
// Phase exponent of gen*key for a raw generator (the frame conjugation uses
// every tableau row as a generator).
template <int W, int ALG>
__device__ int product_exp_raw(const u64* gen, const u64* key) {
  if constexpr (ALG == 0) {
    int yg = 0, yk = 0, yo = 0, zx = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) {
      const u64 o = key[i] ^ gen[i];
      yg += __popcll(gen[i] & (gen[i] >> 1) & EVEN);
      yk += __popcll(key[i] & (key[i] >> 1) & EVEN);
      yo += __popcll(o & (o >> 1) & EVEN);
      zx += __popcll((gen[i] >> 1) & key[i] & EVEN);
    }
    return (yg + yk - yo + 2 * zx) & 3;
  } else {
    int lg = 0, lk = 0, lo = 0, sw = 0;
    u32 above = 0;  // parity of generator modes in higher words
#pragma unroll
    for (int i = W - 1; i >= 0; --i) {
      const u64 o = key[i] ^ gen[i];
      const int pg = __popcll(gen[i]), pk = __popcll(key[i]);
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

// Readout conjugation through a deferred Clifford frame (tableau.rs:93-143):
// fold the rows selected by the key's bits, tracking the phase of the rebuilt
// source and of the image; the sign is -1 iff their ratio is -1.
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
      u64 gk[W];
#pragma unroll
      for (int i = 0; i < W; ++i) gk[i] = __ldg(img + i);
      ie += product_exp_raw<W, ALG>(gk, out) + (signs[p] < 0 ? 2 : 0);
#pragma unroll
      for (int i = 0; i < W; ++i) out[i] ^= gk[i];
    }
  }
  return (((ie - se) & 3) == 2) ? -1.0 : 1.0;
}

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}
__device__ __forceinline__ void dd_add(double& hi, double& lo, double v) {
  double s, e;
  two_sum(hi, v, s, e);
  e = __dadd_rn(e, lo);
  two_sum(s, e, hi, lo);
}

// sum c * <s|frame(K)|s> in double-double, plus the count of |c| < min_coeff
// (partitioned_termsum.rs:611-697).
template <int W, int ALG>
__global__ void __launch_bounds__(BLOCK) expect_kernel(const ExpectArgs a, const u64* keys, const double* coeffs,
                                                       u64 N, ExpectPartial* partials) {
  using Ops = typename Alg<ALG>::T;
  double hi = 0, lo = 0, ab = 0;
  u64 below = 0;
  for (u64 r = (u64)blockIdx.x * BLOCK + threadIdx.x; r < N; r += (u64)gridDim.x * BLOCK) {
    u64 key[W];
    load_key<W>(keys, r, key);
    const double c = coeffs[r];
    if (a.has_min_coeff && fabs(c) < a.min_coeff) ++below;
    double v;
    if (a.frame_images) {
      u64 img[W];
      const double sg = conjugate_key<W, ALG>(key, a.frame_images, a.frame_signs, a.frame_rows, img);
      v = __dmul_rn(__dmul_rn(c, sg), Ops::template trace<W>(img, a.state, a.n_units));
    } else {
      v = __dmul_rn(c, Ops::template trace<W>(key, a.state, a.n_units));
    }
    if (v != 0.0) {
      dd_add(hi, lo, v);
      ab += fabs(v);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ohi = __shfl_xor_sync(FULL, hi, o), olo = __shfl_xor_sync(FULL, lo, o);
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

// ------------------------------------------------------------ adjoint
// Reverse sweep of one recorded segment.  With the truncation decisions of the
// forward run frozen, each op is linear in the coefficients, so dE/dc of its
// input rows is the transpose of the op applied to dE/dc of its output rows:
//   gate, row r anticommuting with G, coefficient c, sin branch to row p:
//     lam_in[r] = cos * lam_out[r] + sin * s_r * lam_out[p]
//     dE/dangle += -sin * c * lam_out[r] + cos * s_r * c * lam_out[p]
//   (s_r = -Im of the phase of G K_r, times the frame sign of G), and
//   lam_in[r] = lam_out[r] for commuting rows;
//   noise: lam_in[r] = f(w_r) * lam_out[new index of r] (0 if dropped).
// lam_out was written by other blocks during the previous op, so it is read
// through L2 (ld.cg).

__device__ __forceinline__ void block_partial(double v, double* out) {
  __shared__ double red[NWARPS];
  for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_xor_sync(FULL, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < NWARPS; ++w) t = __dadd_rn(t, red[w]);
    *out = t;
  }
  __syncthreads();
}

template <int W, int ALG>
__device__ __noinline__ void adjoint_gate(const AdjointArgs& a, const GateDesc<W>& d, u32 op, bool phase, u64 N,
                                          const u64* keys, const double* lin, double* lout) {
  using Ops = typename Alg<ALG>::T;
  const u64 o = a.rec_off[op];
  double gsum = 0.0;
  for (u64 r = (u64)blockIdx.x * BLOCK + threadIdx.x; r < N; r += (u64)gridDim.x * BLOCK) {
    u64 key[W];
    load_key<W>(keys, r, key);
    const double l = __ldcg(lin + r);
    if (!Ops::template anticommutes<W>(d.g, key)) {
      lout[r] = l;
      continue;
    }
    const double c = __ldg(a.rec_coef + o + r);
    double v = __dmul_rn(d.cs, l);
    gsum = __dadd_rn(gsum, -__dmul_rn(__dmul_rn(d.sn, c), l));
    const u32 p = phase ? REC_NONE : __ldg(a.rec_idx + o + r);
    if (p != REC_NONE) {
      const double sr = neg_im(Ops::template product_exp<W>(d.g, key), d.g.sign);
      const double lp = __ldcg(lin + p);
      v = __dadd_rn(v, __dmul_rn(__dmul_rn(d.sn, sr), lp));
      gsum = __dadd_rn(gsum, __dmul_rn(__dmul_rn(__dmul_rn(d.cs, sr), c), lp));
    }
    lout[r] = v;
  }
  block_partial(gsum, a.grad_part + (u64)op * gridDim.x + blockIdx.x);
}

template <int W, int ALG>
__device__ __noinline__ void adjoint_noise(const AdjointArgs& a, const double* factors, u32 op, bool compact, u64 N,
                                           const u64* keys, const double* lin, double* lout) {
  using Ops = typename Alg<ALG>::T;
  const u32 last = a.table_len - 1;
  const u64 o = a.rec_off[op];
  for (u64 r = (u64)blockIdx.x * BLOCK + threadIdx.x; r < N; r += (u64)gridDim.x * BLOCK) {
    u64 key[W];
    load_key<W>(keys, r, key);
    const u32 w = Ops::template weight<W>(key, a.n_units);
    const double f = __ldg(factors + (w < last ? w : last));
    if (compact) {
      const u32 p = __ldg(a.rec_idx + o + r);
      lout[r] = p == REC_NONE ? 0.0 : __dmul_rn(f, __ldcg(lin + p));
    } else {
      lout[r] = __dmul_rn(f, __ldcg(lin + r));
    }
  }
}

template <int W, int ALG>
__global__ void __launch_bounds__(BLOCK, MinBlocks<W>::value) adjoint_kernel(const AdjointArgs a) {
  __shared__ GateDesc<W> sgate;
  const Grp grp{blockIdx.x, gridDim.x};
  SweepState* st = a.st;
  u32 gen = *(volatile u32*)&st->bar_gen;
  int cur = (int)a.cur0;
  for (u32 op = a.op_end; op-- > a.op_begin;) {
    const OpDesc od = a.ops[op];
    const u64 N = a.n_in[op];
    const u64* keys = a.key_src[op];
    const double* lin = a.lam[cur];
    double* lout = a.lam[cur ^ 1];
    if (od.kind == OP_GATE || od.kind == OP_PHASE) {
      if (threadIdx.x == 0) sgate = reinterpret_cast<const GateDesc<W>*>(a.gates)[od.idx];
      __syncthreads();
      adjoint_gate<W, ALG>(a, sgate, op, od.kind == OP_PHASE, N, keys, lin, lout);
    } else {
      adjoint_noise<W, ALG>(a, a.tables + (u64)od.idx * a.table_len, op, od.kind == OP_NOISE_COMPACT, N, keys, lin,
                            lout);
    }
    cur ^= 1;
    grid_barrier(st, gen, grp);
    if (*(volatile u32*)&st->error) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st->cur = (u32)cur;
}

template <int W, int ALG>
__global__ void adjoint_seed_kernel(const ExpectArgs a, const u64* keys, u64 N, double* lam) {
  using Ops = typename Alg<ALG>::T;
  for (u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (u64)gridDim.x * blockDim.x) {
    u64 key[W];
    load_key<W>(keys, r, key);
    if (a.frame_images) {
      u64 img[W];
      const double sg = conjugate_key<W, ALG>(key, a.frame_images, a.frame_signs, a.frame_rows, img);
      lam[r] = __dmul_rn(sg, Ops::template trace<W>(img, a.state, a.n_units));
    } else {
      lam[r] = Ops::template trace<W>(key, a.state, a.n_units);
    }
  }
}

__global__ void grad_reduce_kernel(const double* grad_part, int grid, const long long* gate_ops, u64 n_gates,
                                   double* grad) {
  for (u64 g = (u64)blockIdx.x * blockDim.x + threadIdx.x; g < n_gates; g += (u64)gridDim.x * blockDim.x) {
    const long long op = gate_ops[g];
    if (op < 0) {
      grad[g] = __longlong_as_double(0x7ff8000000000000LL);  // quiet NaN: no op of its own
      continue;
    }
    double t = 0.0;
    for (int b = 0; b < grid; ++b) t = __dadd_rn(t, grad_part[(u64)op * grid + b]);
    grad[g] = t;
  }
}

template <int W>
__global__ void rebuild_kernel(const u64* keys, u64 N, u64* table, u64 mask, u64 bmask, u32* error) {
  for (u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (u64)gridDim.x * blockDim.x) {
    u64 key[W];
    load_key<W>(keys, r, key);
    insert<W>(key, r, table, mask, bmask, error);
  }
}

template <int W, int ALG>
__global__ void conjugate_kernel(const u64* keys, const double* coeffs, u64 n, const u64* images, const int* signs,
                                 u32 rows, u64* out_keys, double* out_coeffs) {
  for (u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (u64)gridDim.x * blockDim.x) {
    u64 key[W], img[W];
    load_key<W>(keys, r, key);
    const double sg = conjugate_key<W, ALG>(key, images, signs, rows, img);
    store_key<W>(out_keys, r, img);
    out_coeffs[r] = __dmul_rn(coeffs[r], sg);
  }
}

}  // namespace

// Blocks of `k` that fit on every SM at once (the grid of a cooperative
// launch).  Once per kernel it also asks for the smallest shared-memory share
// of the SM's unified L1 / shared memory that keeps that many blocks
// resident: the sweeps are chains of dependent loads, and the rest of the
// 256 KB is L1 for their rows, descriptors and local memory.  If the smaller
// share would cost a resident block, the driver's default stays.
template <class Kernel>
int co_resident_grid(Kernel k, int blocks_per_sm, int* sms, int* per_sm) {
  if (!*sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, dev);
    int p = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, k, BLOCK, 0);
    int smem_sm = 0, reserved = 0;
    cudaFuncAttributes fa{};
    if (p > 0 && cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) == cudaSuccess &&
        cudaFuncGetAttributes(&fa, k) == cudaSuccess && smem_sm > 0) {
      const size_t need = (size_t)p * (fa.sharedSizeBytes + (size_t)reserved);
      const int pct = (int)((need * 100 + (size_t)smem_sm - 1) / (size_t)smem_sm);
      if (pct < 100 && cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, pct) == cudaSuccess) {
        int p2 = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p2, k, BLOCK, 0);
        if (p2 < p) cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, -1);
      }
      cudaGetLastError();  // a refused hint is not an error of the run
    }
    *per_sm = p < 1 ? 1 : p;
  }
  const int b = (blocks_per_sm > 0 && blocks_per_sm < *per_sm) ? blocks_per_sm : *per_sm;
  return *sms * b;
}

template <int W, int ALG>
int sweep_grid(int blocks_per_sm, int build) {
  if constexpr (W <= 2) {
    if (build == SWEEP_SIX) {
      static int sms = 0, per_sm = 0;
      return co_resident_grid(sweep_kernel_occ<W, ALG>, blocks_per_sm, &sms, &per_sm);
    }
  }
  if constexpr (W <= 4) {
    if (build == SWEEP_TWO) {
      static int sms = 0, per_sm = 0;
      return co_resident_grid(sweep_kernel_two<W, ALG>, blocks_per_sm, &sms, &per_sm);
    }
  }
  static int sms = 0, per_sm = 0;
  return co_resident_grid(sweep_kernel<W, ALG>, blocks_per_sm, &sms, &per_sm);
}

template <int WM, int ALG>
int batch_grid(int blocks_per_sm) {
  static int sms = 0, per_sm = 0;
  return co_resident_grid(batch_sweep_kernel<WM, ALG>, blocks_per_sm, &sms, &per_sm);
}

template <int W, int ALG>
cudaError_t launch_sweep(const SweepArgs& a, int grid, cudaStream_t s, int build) {
  SweepArgs args = a;
  void* params[] = {&args};
  const void* k = (const void*)sweep_kernel<W, ALG>;
  if constexpr (W <= 2) {
    if (build == SWEEP_SIX) k = (const void*)sweep_kernel_occ<W, ALG>;
  }
  if constexpr (W <= 4) {
    if (build == SWEEP_TWO) k = (const void*)sweep_kernel_two<W, ALG>;
  }
  return cudaLaunchCooperativeKernel(k, dim3(grid), dim3(BLOCK), params, 0, s);
}

template <int W, int ALG>
cudaError_t launch_batch_sweep(const SweepArgs* args, const u32* block_inst, int grid, cudaStream_t s) {
  void* params[] = {(void*)&args, (void*)&block_inst};
  return cudaLaunchCooperativeKernel((const void*)batch_sweep_kernel<W, ALG>, dim3(grid), dim3(BLOCK), params, 0,
                                     s);
}

template <int W, int ALG>
cudaError_t launch_adjoint(const AdjointArgs& a, int grid, cudaStream_t s) {
  AdjointArgs args = a;
  void* params[] = {&args};
  return cudaLaunchCooperativeKernel((const void*)adjoint_kernel<W, ALG>, dim3(grid), dim3(BLOCK), params, 0, s);
}

template <int W, int ALG>
cudaError_t launch_adjoint_seed(const ExpectArgs& a, const u64* keys, u64 n, double* lam, cudaStream_t s) {
  if (!n) return cudaSuccess;
  const int threads = 256;
  const u64 blocks = (n + threads - 1) / threads;
  adjoint_seed_kernel<W, ALG><<<(unsigned)(blocks < 65535 ? blocks : 65535), threads, 0, s>>>(a, keys, n, lam);
  return cudaGetLastError();
}

#ifndef PQ_ONLY_WIDTH  // defined once, in the translation unit of the narrow widths
cudaError_t launch_grad_reduce(const double* grad_part, int grid, const long long* gate_ops, u64 n_gates,
                               double* grad, cudaStream_t s) {
  if (!n_gates) return cudaSuccess;
  const u64 blocks = (n_gates + 255) / 256;
  grad_reduce_kernel<<<(unsigned)(blocks < 65535 ? blocks : 65535), 256, 0, s>>>(grad_part, grid, gate_ops, n_gates,
                                                                                  grad);
  return cudaGetLastError();
}
#endif

template <int W, int ALG>
int adjoint_grid() {
  static int sms = 0, per_sm = 0;
  return co_resident_grid(adjoint_kernel<W, ALG>, 0, &sms, &per_sm);
}

template <int W, int ALG>
cudaError_t launch_expect(const ExpectArgs& a, const u64* keys, const double* coeffs, u64 n,
                          ExpectPartial* partials, int grid, cudaStream_t s) {
  expect_kernel<W, ALG><<<grid, BLOCK, 0, s>>>(a, keys, coeffs, n, partials);
  return cudaGetLastError();
}

template <int W>
cudaError_t launch_rebuild(const u64* keys, u64 n, u64* table, u64 mask, u64 bmask, u32* error, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const u64 blocks = (n + 255) / 256;
  rebuild_kernel<W><<<(int)(blocks < 8192 ? blocks : 8192), 256, 0, s>>>(keys, n, table, mask, bmask, error);
  return cudaGetLastError();
}

template <int W>
cudaError_t launch_conjugate(const u64* keys, const double* coeffs, u64 n, const u64* images, const int* signs,
                             u32 rows, int alg, u64* out_keys, double* out_coeffs, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const u64 blocks = (n + 255) / 256;
  const int grid = (int)(blocks < 4096 ? blocks : 4096);
  if (alg == 0)
    conjugate_kernel<W, 0><<<grid, 256, 0, s>>>(keys, coeffs, n, images, signs, rows, out_keys, out_coeffs);
  else
    conjugate_kernel<W, 1><<<grid, 256, 0, s>>>(keys, coeffs, n, images, signs, rows, out_keys, out_coeffs);
  return cudaGetLastError();
}

#define PQ_INSTANTIATE(Wv, Av)                                                                          \
  template int sweep_grid<Wv, Av>(int, int);                                                              \
  template int batch_grid<Wv, Av>(int);                                                                    \
  template cudaError_t launch_sweep<Wv, Av>(const SweepArgs&, int, cudaStream_t, int);                 \
  template cudaError_t launch_batch_sweep<Wv, Av>(const SweepArgs*, const u32*, int, cudaStream_t);     \
  template cudaError_t launch_adjoint<Wv, Av>(const AdjointArgs&, int, cudaStream_t);                   \
  template cudaError_t launch_adjoint_seed<Wv, Av>(const ExpectArgs&, const u64*, u64, double*, cudaStream_t); \
  template int adjoint_grid<Wv, Av>();                                                                  \
  template cudaError_t launch_expect<Wv, Av>(const ExpectArgs&, const u64*, const double*, u64,         \
                                             ExpectPartial*, int, cudaStream_t);
#define PQ_INSTANTIATE_KEYS(Wv)                                                                         \
  template cudaError_t launch_rebuild<Wv>(const u64*, u64, u64*, u64, u64, u32*, cudaStream_t);         \
  template cudaError_t launch_conjugate<Wv>(const u64*, const double*, u64, const u64*, const int*, u32, int, \
                                            u64*, double*, cudaStream_t);
#define PQ_INSTANTIATE_W(Wv)                                                                            \
  PQ_INSTANTIATE(Wv, 0)                                                                                 \
  PQ_INSTANTIATE(Wv, 1)                                                                                 \
  PQ_INSTANTIATE_KEYS(Wv)

// Key widths 1 and 2 words (up to 64 units) here; 4, 8, 16, 32 and 64 words
// each in a translation unit of its own (pq_kernels_w4.cu ...) that defines
// PQ_ONLY_WIDTH and includes this file, so that the widths compile in
// parallel.  The 32- and 64-word kernels, the slowest to compile, are split
// further by algebra: pq_kernels_w64.cu also defines PQ_ONLY_ALG 0 (Pauli,
// with the algebra-free key kernels), pq_kernels_w64_majorana.cu PQ_ONLY_ALG 1.
#if defined(PQ_ONLY_WIDTH) && defined(PQ_ONLY_ALG)
PQ_INSTANTIATE(PQ_ONLY_WIDTH, PQ_ONLY_ALG)
#if PQ_ONLY_ALG == 0
PQ_INSTANTIATE_KEYS(PQ_ONLY_WIDTH)
#endif
#elif defined(PQ_ONLY_WIDTH)
PQ_INSTANTIATE_W(PQ_ONLY_WIDTH)
#else
PQ_INSTANTIATE_W(1)
PQ_INSTANTIATE_W(2)
#endif

}  // namespace pq
