// pq_class.cuh -- the class op of the sweep: m rotations in one op.
//
// Included by pq_kernels.cu inside its anonymous namespace (it uses that
// file's barrier, look-back, lookup and placement helpers).
//
// A class is a run of m rotations G_0..G_{m-1} (Heisenberg order) of the Pauli
// basis whose generators act on pairwise disjoint qubits, so they commute and
// each has a "pivot" key bit that no other generator of the class has.  For a
// row K let S(K) be the class rotations K anticommutes with (k = |S| of them).
// Every key K ^ G_j1 ^ ... (j in S) anticommutes with exactly the same
// rotations, and no rotation of the class moves a term outside that set, so
// the reference's gate-by-gate steps (crates/core/src/engine/termsum.rs:
// 604-751, one rotation after the other) act on each such set -- a family, a
// k-cube of keys indexed by their pivot bits -- independently of every other
// family.  The class op therefore runs each family through all of its
// rotations at once, in gate order, with the reference's pair rule at every
// step: every coefficient is the same two-operand result as in m separate
// ops, the per-gate live counts are the same, and only the positions at which
// new rows are appended differ (deterministically: by owner row, then by the
// member's pivot code).
//
// Three phases, with a grid barrier after each of the first two:
//   A  every row: its class mask S; rows with S != 0 join their family in the
//      family table (keyed by the family's representative, the member with no
//      pivot bit set), counting the family's present members and its least
//      row, the family's owner;
//   B  every owner: run the family and count the rows it creates, per gate and
//      in total; a block scan and the decoupled look-back give each tile's
//      offset; the last tile publishes the live count after the class.  A
//      class that would pass the row capacity stops here, before any write
//      (the host grows the buffers and runs it again);
//   C  every owner: run the family again and write it: the coefficients of
//      its present members and its new rows, in order, inserted into the hash
//      table; the owner clears its family slot.
// A family with one present member runs in the owner's thread (no two of its
// members meet within a class) while it takes at most LONE_BUDGET member
// steps; larger or multi-member families run on the owner's warp, 2^k members
// spread over the lanes (k <= FAM_KMAX).  The host forms
// classes only where k <= FAM_KMAX holds for every live row (a weight cut of
// at most FAM_KMAX keeps every row's weight, hence k, within it); a row beyond
// it all the same raises ERR_CLASS_FAMILY.
#pragma once

constexpr int FAM_KMAX = (int)CLASS_KMAX;  // largest family dimension a class op runs
constexpr int LONE_BUDGET = 256;  // member steps a single-member family may take in one thread
constexpr int WARP_SLOTS = (1 << FAM_KMAX) / 32;  // members per lane on the warp path

struct ClassSmem {
  u32 children[CLASS_MAX];  // rows created per rotation of the class (this block)
  u32 anti[CLASS_MAX];      // rows anticommuting per rotation (this block)
  u32 wsum[NWARPS];         // block scan
  u32 tile_excl;
  u32 tile_agg;
};

// Key of family member `code` (bit i: times the class rotation sidx[i]).
template <int W>
__device__ __forceinline__ void member_key(const u64* rep, const GateDesc<W>* cg, const int* sidx, u32 code,
                                           u64* out) {
#pragma unroll
  for (int w = 0; w < W; ++w) out[w] = rep[w];
  for (u32 c = code; c; c &= c - 1) {
    const u64* g = cg[sidx[__ffs(c) - 1]].g.gen;
#pragma unroll
    for (int w = 0; w < W; ++w) out[w] ^= g[w];
  }
}

__device__ __forceinline__ bool key_bit(const u64* k, u32 bit) { return (k[bit >> 6] >> (bit & 63)) & 1ull; }

// The class rotations a key anticommutes with (bit j = rotation j).  For
// Pauli keys from `fold`, the class's pair-swapped generators (W words each)
// in shared memory: the one part of the descriptors every row reads.
template <int W, int ALG>
__device__ __forceinline__ u64 class_mask(const u64* key, const GateDesc<W>* cg, const u64* fold, u32 m) {
  u64 s = 0;
  if constexpr (ALG == 0) {
    for (u32 j = 0; j < m; ++j) {
      u64 acc = 0;
#pragma unroll
      for (int w = 0; w < W; ++w) acc ^= key[w] & fold[j * W + w];
      if (popc(acc) & 1) s |= 1ull << j;
    }
  } else {
    using Ops = typename Alg<ALG>::T;
    for (u32 j = 0; j < m; ++j)
      if (Ops::template anticommutes<W>(cg[j].g, key)) s |= 1ull << j;
  }
  return s;
}

// The family's representative (its member with no pivot bit set), the list of
// its rotations in gate order, and the pivot code of `key` itself.
template <int W>
__device__ __forceinline__ int family_of(const u64* key, u64 S, const GateDesc<W>* cg, u64* rep, int* sidx,
                                         u32& code) {
  int k = 0;
  code = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) rep[w] = key[w];
  for (u64 s = S; s && k < FAM_KMAX; s &= s - 1, ++k) {
    const int j = __ffsll((long long)s) - 1;
    sidx[k] = j;
    if (key_bit(key, cg[j].pivot)) {
      code |= 1u << k;
#pragma unroll
      for (int w = 0; w < W; ++w) rep[w] ^= cg[j].g.gen[w];
    }
  }
  return __popcll(S);
}

// The emit rules of one step of the class (the same as gate_tiles).
template <int W, int ALG>
struct ClassRules {
  using Ops = typename Alg<ALG>::T;
  u32 wcut, n_units;
  bool ccut;
  double minc;
  __device__ __forceinline__ int state(double c, const u64* child, const GateDesc<W>& d) const {
    if (ccut && fabs(__dmul_rn(c, d.sn)) < minc) return S_HELD;
    if (wcut != NO_WEIGHT_CUT && Ops::template weight<W>(child, n_units) > wcut) return S_DROP;
    return S_EMIT;
  }
  __device__ __forceinline__ double branch(double c, const u64* key, const GateDesc<W>& d) const {
    return __dmul_rn(__dmul_rn(c, d.sn), neg_im(Ops::template product_exp<W>(d.g, key), d.g.sign));
  }
};

// A family whose only present member is its owner row, in one thread.  No
// two members can meet within the class: a member present at step i differs
// from the owner only in pivot bits of earlier steps, while its partner at
// step i differs in pivot bit i, which only step i sets.  So every member
// evolves on its own -- at each later step its cos branch stays and its sin
// branch becomes a new member on EMIT -- and the family is walked depth
// first, a new member before the rest of its parent's steps, with the
// members numbered as they are created.  WRITE = false counts (per step into
// nchild / nanti, and the total); WRITE = true writes the owner's final
// coefficient and each new member at base + its number.  False (nothing
// written) if the walk passes `budget` member steps; the warp path then runs
// the family.
template <int W, int ALG, bool WRITE>
__device__ bool run_lone(const ClassRules<W, ALG>& R, const u64* key0, const int* sidx, int k, double c0,
                         const GateDesc<W>* cg, int budget, u32* nchild, u32* nanti, u32& n_new,
                         const SweepArgs& a, u64 r, u64 base, u64* keys, double* coeffs) {
  struct Frame {
    u32 code;  // pivot bits flipped relative to the owner
    u32 step;  // next step to apply
    u32 num;   // 0 = the owner, else 1 + the member's creation number
    double c;
  };
  Frame stack[FAM_KMAX];
  int depth = 0;
  Frame cur{0u, 0u, 0u, c0};
  u64 key[W];
#pragma unroll
  for (int w = 0; w < W; ++w) key[w] = key0[w];
  n_new = 0;
  int work = 0;
  for (;;) {
    for (u32 i = cur.step; i < (u32)k; ++i) {
      if (++work > budget) return false;
      const GateDesc<W>& d = cg[sidx[i]];
      if (!WRITE) ++nanti[i];
      u64 child[W];
#pragma unroll
      for (int w = 0; w < W; ++w) child[w] = key[w] ^ d.g.gen[w];
      const double b = R.branch(cur.c, key, d);
      const int st = R.state(cur.c, child, d);
      cur.c = __dmul_rn(cur.c, d.cs);
      if (st == S_EMIT) {  // the new member first, the parent resumes at step i + 1
        if (!WRITE) ++nchild[i];
        stack[depth++] = Frame{cur.code, i + 1, cur.num, cur.c};
        cur = Frame{cur.code ^ (1u << i), i + 1, ++n_new, b};
#pragma unroll
        for (int w = 0; w < W; ++w) key[w] = child[w];
      }
    }
    if (WRITE) {
      if (cur.num == 0) {
        coeffs[r] = cur.c;
      } else {
        const u64 row = base + cur.num - 1;
        if (row < a.cap) {
          store_key<W>(keys, row, key);
          coeffs[row] = cur.c;
          insert<W>(key, row, a.table, a.table_mask, a.table_bmask, &a.st->error);
        } else {
          atomicOr(&a.st->error, ERR_CAPACITY);
        }
      }
    }
    if (depth == 0) return true;
    cur = stack[--depth];
    // the parent's key: the owner's with its flipped pivots' generators
#pragma unroll
    for (int w = 0; w < W; ++w) key[w] = key0[w];
    for (u32 c = cur.code; c; c &= c - 1) {
      const u64* g = cg[sidx[__ffs(c) - 1]].g.gen;
#pragma unroll
      for (int w = 0; w < W; ++w) key[w] ^= g[w];
    }
  }
}

// A family on the owner's warp: member c = lane + 32 s (s < slots) of the
// 2^k-cube.  Every lane looks its members up among the rows entering the op
// (row, coefficient, and the empty slot a miss ended on), then each step
// updates every member from its own and its partner's values before the step
// (the partner is in lane ^ 2^i for i < 5, else slot s ^ 2^(i-5) of the same
// lane), so that each lane writes only its own members.  `orig` marks members
// present at entry, `pres` those present at the end.
template <int W, int ALG>
struct WarpFamily {
  double cf[WARP_SLOTS];
  u32 row[WARP_SLOTS];
  u64 slot[WARP_SLOTS];
  u32 pres, orig;
  int slots;
};

template <int W, int ALG>
__device__ __noinline__ void run_warp_family(const ClassRules<W, ALG>& R, const SweepArgs& a, u64 N,
                                             const u64* keys, const double* coeffs, const u64* rep, const int* sidx,
                                             int k, const GateDesc<W>* cg, WarpFamily<W, ALG>& F, ClassSmem& cs,
                                             bool count) {
  const int lane = threadIdx.x & 31;
  const u32 size = 1u << k;
  F.slots = size > 32 ? (int)(size >> 5) : 1;
  F.pres = 0;
  for (int s = 0; s < F.slots; ++s) {
    const u32 c = (u32)lane + 32u * (u32)s;
    F.cf[s] = 0.0;
    F.row[s] = REC_NONE;
    F.slot[s] = NO_SLOT;
    if (c >= size) continue;
    u64 q[W];
    member_key<W>(rep, cg, sidx, c, q);
    double cj = 0.0;
    u64 es = NO_SLOT;
    const long long j = lookup_c<W>(q, N, keys, coeffs, a.table, a.table_mask, a.table_bmask, a.st, cj, es, 0);
    if (j >= 0) {
      F.pres |= 1u << s;
      F.cf[s] = cj;
      F.row[s] = (u32)j;
    } else {
      F.slot[s] = es;
    }
  }
  F.orig = F.pres;
  for (int i = 0; i < k; ++i) {
    const GateDesc<W>& d = cg[sidx[i]];
    u32 np = F.pres;
    double ncf[WARP_SLOTS];
    for (int s = 0; s < F.slots; ++s) ncf[s] = F.cf[s];
    if (count) {
      const u32 na = __reduce_add_sync(FULL, (u32)__popc(F.pres));
      if (lane == 0 && na) atomicAdd(&cs.anti[sidx[i]], na);
    }
    for (int s = 0; s < F.slots; ++s) {
      const u32 c = (u32)lane + 32u * (u32)s;
      int ps;
      double pc;
      bool pp;
      if (i < 5) {  // the partner is in another lane, same slot
        ps = s;
        pc = __shfl_xor_sync(FULL, F.cf[s], 1 << i);
        pp = (__shfl_xor_sync(FULL, F.pres, 1 << i) >> s) & 1u;
      } else {
        ps = s ^ (1 << (i - 5));
        pc = F.cf[ps];
        pp = (F.pres >> ps) & 1u;
      }
      const bool pm = (F.pres >> s) & 1u;
      if (c >= size || (!pm && !pp)) continue;
      u64 km[W], kp[W];
      member_key<W>(rep, cg, sidx, c, km);
#pragma unroll
      for (int w = 0; w < W; ++w) kp[w] = km[w] ^ d.g.gen[w];
      const double cm = F.cf[s];
      if (pm && pp) {
        const double bp = R.branch(pc, kp, d);
        const int sm = R.state(cm, kp, d), sp = R.state(pc, km, d);
        const bool to_m = sp == S_EMIT || (sp == S_HELD && sm == S_EMIT);
        double v = __dmul_rn(cm, d.cs);
        if (to_m) v = __dadd_rn(v, bp);
        ncf[s] = v;
      } else if (pm) {
        ncf[s] = __dmul_rn(cm, d.cs);
      } else if (R.state(pc, km, d) == S_EMIT) {  // the lone partner's sin branch creates this member
        ncf[s] = R.branch(pc, kp, d);
        np |= 1u << s;
      }
    }
    if (count) {
      const u32 born = __reduce_add_sync(FULL, (u32)__popc(np & ~F.pres));
      if (lane == 0 && born) atomicAdd(&cs.children[sidx[i]], born);
    }
    F.pres = np;
    for (int s = 0; s < F.slots; ++s) F.cf[s] = ncf[s];
  }
}

// Rank of each new member in pivot-code order (code = lane + 32 s): the
// members of lower slots, then those of lower lanes in the same slot.
template <int W, int ALG>
__device__ __forceinline__ void write_warp_family(const SweepArgs& a, const u64* rep, const int* sidx,
                                                  const GateDesc<W>* cg, const WarpFamily<W, ALG>& F, u64 base,
                                                  u64* keys, double* coeffs) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  u64 before = 0;
  for (int s = 0; s < F.slots; ++s) {
    const bool o = (F.orig >> s) & 1u, p = (F.pres >> s) & 1u;
    if (o) coeffs[F.row[s]] = F.cf[s];
    const unsigned bm = __ballot_sync(FULL, p && !o);
    if (p && !o) {
      const u64 row = base + before + __popc(bm & lt);
      if (row < a.cap) {
        u64 q[W];
        member_key<W>(rep, cg, sidx, (u32)lane + 32u * (u32)s, q);
        store_key<W>(keys, row, q);
        coeffs[row] = F.cf[s];
        place_from<W>(q, ((key_hash<W>(q) >> 32) << 32) | (row & 0xffffffffULL), F.slot[s], a.table,
                      a.table_mask, a.table_bmask, &a.st->error);
      } else {
        atomicOr(&a.st->error, ERR_CAPACITY);
      }
    }
    before += __popc(bm);
  }
}

// Block-wide exclusive scan of one count per thread; returns this thread's
// offset and leaves the block's total in cs.tile_agg.
__device__ __forceinline__ u32 block_excl_scan(u32 v, ClassSmem& cs) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u32 inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u32 y = __shfl_up_sync(FULL, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) cs.wsum[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const u32 w = lane < NWARPS ? cs.wsum[lane] : 0u;
    u32 wi = w;
#pragma unroll
    for (int o = 1; o < NWARPS; o <<= 1) {
      const u32 y = __shfl_up_sync(FULL, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < NWARPS) cs.wsum[lane] = wi - w;
    if (lane == NWARPS - 1) cs.tile_agg = wi;
  }
  __syncthreads();
  return cs.wsum[warp] + inc - v;
}

// Phase A for the rows of this block: class masks and family membership.
template <int W, int ALG>
__device__ __noinline__ void class_phase_a(const SweepArgs& a, const GateDesc<W>* cg, const u64* fold, u32 m, u32 op,
                                           u64 N, const u64* keys, const Grp grp) {
  SweepState* st = a.st;
  for (u64 r = (u64)grp.bid * BLOCK + threadIdx.x; r < N; r += (u64)grp.nblk * BLOCK) {
    u64 key[W];
    load_key<W>(keys, r, key);
    const u64 S = class_mask<W, ALG>(key, cg, fold, m);
    a.cls_mask[r] = S;
    if (!S) continue;
    u64 rep[W];
    int sidx[FAM_KMAX];
    u32 code;
    const int k = family_of<W>(key, S, cg, rep, sidx, code);
    if (k > FAM_KMAX) {  // ruled out by the host's choice of classes
      atomicOr(&st->error, ERR_CLASS_FAMILY);
      a.cls_slot[r] = REC_NONE;
      continue;
    }
    // join the family: its representative's slot (fingerprint, first row); a
    // fingerprint match is the same family iff the two keys differ by
    // rotations of this family
    const u64 h = key_hash<W>(rep);
    const u32 fp = (u32)(h >> 32);
    const u64 want = ((u64)fp << 32) | (u32)r;
    u64 i = (h & a.table_mask) & ~3ULL;  // buckets of 4 slots
    u64 found = NO_SLOT;
    for (u64 probe = 0; probe <= a.table_mask; ++probe) {
      u64 s = __ldcg(a.fam_table + i);
      if (s == EMPTY_SLOT) {
        s = atomicCAS(a.fam_table + i, EMPTY_SLOT, want);
        if (s == EMPTY_SLOT) {
          found = i;
          break;
        }
      }
      if ((u32)(s >> 32) == fp) {
        u64 d[W];
        load_key<W>(keys, (u32)s, d);
#pragma unroll
        for (int w = 0; w < W; ++w) d[w] ^= rep[w];
        for (int t = 0; t < k; ++t)
          if (key_bit(d, cg[sidx[t]].pivot)) {
#pragma unroll
            for (int w = 0; w < W; ++w) d[w] ^= cg[sidx[t]].g.gen[w];
          }
        u64 z = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) z |= d[w];
        if (!z) {
          found = i;
          break;
        }
      }
      i = (i + 1) & a.table_mask;
    }
    if (found == NO_SLOT) {
      atomicOr(&st->error, ERR_PROBE_OVERFLOW);
      a.cls_slot[r] = REC_NONE;
      continue;
    }
    a.cls_slot[r] = (u32)found;
    u32* aux = reinterpret_cast<u32*>(a.fam_aux + found);  // [~least row, count]
    atomicMax(aux, ~(u32)r);
    atomicAdd(aux + 1, 1u);
  }
}

// Phases B (count) and C (write) for one row of a tile: returns the rows its
// family creates (0 unless the row owns its family), with WARP_PATH set if the
// family ran on the warp path.  Phase C passes phase B's answer back in
// `path` (so both phases take the same path) and the row's first new row,
// base_in_tile + my_off.
constexpr u32 WARP_PATH = 0x80000000u;
template <int W, int ALG, bool WRITE>
__device__ __noinline__ u32 class_tile(const SweepArgs& a, const ClassRules<W, ALG>& R, const GateDesc<W>* cg,
                                       u64 N, u64 r, u64* keys, double* coeffs, ClassSmem& cs, u64 base_in_tile,
                                       u32 my_off, u32 path) {
  const int lane = threadIdx.x & 31;
  // 0: nothing to do; 1: a lone family run here; 2: a family for the warp path
  int mode = 0;
  u64 key[W], rep[W];
  int sidx[FAM_KMAX];
  u32 code = 0;
  int k = 0;
  double c0 = 0.0;
  u32 children = 0;
  if (r < N) {
    const u64 S = a.cls_mask[r];
    const u32 slot = S ? a.cls_slot[r] : REC_NONE;
    if (slot != REC_NONE) {  // (REC_NONE: the row found no family slot and raised an error)
      const u64 aux = __ldcg(a.fam_aux + slot);
      if (~(u32)aux == (u32)r) {  // the family's least row owns it
        load_key<W>(keys, r, key);
        k = family_of<W>(key, S, cg, rep, sidx, code);
        mode = 2;
        if ((u32)(aux >> 32) == 1u && !(WRITE && (path & WARP_PATH))) {  // the owner is the only present member
          c0 = __ldcg(coeffs + r);
          u32 nchild[FAM_KMAX], nanti[FAM_KMAX];
          for (int i = 0; i < FAM_KMAX; ++i) nchild[i] = nanti[i] = 0;
          u32 n_new = 0;
          if (run_lone<W, ALG, WRITE>(R, key, sidx, k, c0, cg, LONE_BUDGET, nchild, nanti, n_new, a, r,
                                       base_in_tile + my_off, keys, coeffs)) {
            mode = 1;
            children = n_new;
            if (!WRITE)
              for (int i = 0; i < k; ++i) {
                if (nchild[i]) atomicAdd(&cs.children[sidx[i]], nchild[i]);
                if (nanti[i]) atomicAdd(&cs.anti[sidx[i]], nanti[i]);
              }
          }
        }
      }
    }
  }
  // the warp path, one family at a time in lane order
  unsigned wm = __ballot_sync(FULL, mode == 2);
  while (wm) {
    const int src = __ffs(wm) - 1;
    wm &= wm - 1;
    u64 frep[W];
#pragma unroll
    for (int w = 0; w < W; ++w) frep[w] = __shfl_sync(FULL, rep[w], src);
    int fsidx[FAM_KMAX];
    const int fk = __shfl_sync(FULL, k, src);
    for (int t = 0; t < FAM_KMAX; ++t) fsidx[t] = __shfl_sync(FULL, sidx[t], src);
    WarpFamily<W, ALG> F;
    run_warp_family<W, ALG>(R, a, N, keys, coeffs, frep, fsidx, fk, cg, F, cs, !WRITE);
    const u32 born = __reduce_add_sync(FULL, (u32)__popc(F.pres & ~F.orig));
    if (lane == src) children = born | WARP_PATH;
    if (WRITE) {
      const u64 base = base_in_tile + __shfl_sync(FULL, my_off, src);
      write_warp_family<W, ALG>(a, frep, fsidx, cg, F, base, keys, coeffs);
    }
  }
  if (WRITE && mode != 0) {  // the family is done: free its slot for the next class
    const u32 slot = a.cls_slot[r];
    a.fam_table[slot] = EMPTY_SLOT;
    a.fam_aux[slot] = 0;
  }
  return children;
}

// The class op: rotations op .. op + m - 1 (their GateDescs at gd).  Returns
// 0 when done, 2 if the class stopped for capacity before any write
// (st->halt and st->need_rows are set), 1 on a device error (the error bits
// end the sweep at the next barrier).
template <int W, int ALG>
__device__ __noinline__ int class_op(const SweepArgs& a, const GateDesc<W>* gd, u32 m, u32 op, u64 N, u64* keys,
                                     double* coeffs, TileSmem& sm, const Grp grp, u64* n_out, u32& gen) {
  // The class's rotations are read where the host put them (through L1),
  // except the pair-swapped generators every row's class mask reads: a shared
  // copy of up to 64 whole descriptors took 6-12 KB of every block's L1 for
  // all ops of every sweep, class or not (the gradient's forward runs, which
  // form no class, went 67.7 -> 72.1 ms).
  const GateDesc<W>* cg = gd;
  __shared__ u64 fold[ALG == 0 ? CLASS_MAX * W : 1];
  __shared__ ClassSmem cs;
  SweepState* st = a.st;
  for (u32 i = threadIdx.x; i < m * W; i += BLOCK) fold[i] = __ldg(&gd[i / W].g.fold[i % W]);
  for (u32 j = threadIdx.x; j < CLASS_MAX; j += BLOCK) {
    cs.children[j] = 0;
    cs.anti[j] = 0;
  }
  __syncthreads();
  class_phase_a<W, ALG>(a, cg, fold, m, op, N, keys, grp);
  grid_barrier(st, gen, grp);
  if (*(volatile u32*)&st->error) return 1;  // the host re-clears the family table after a failed run
  ClassRules<W, ALG> R;
  R.wcut = a.max_weight;
  R.n_units = a.n_units;
  R.ccut = a.has_min_coeff != 0;
  R.minc = a.min_coeff;
  const u32 ntiles = (u32)((N + BLOCK - 1) / BLOCK);
  const u32 epoch = a.epoch_base + op;
  // B: count
  for (u32 t = grp.bid; t < ntiles; t += grp.nblk) {
    const u64 r = (u64)t * BLOCK + threadIdx.x;
    const u32 c = class_tile<W, ALG, false>(a, R, cg, N, r, keys, coeffs, cs, 0, 0u, 0u);
    if (r < N) a.cls_children[r] = c;
    block_excl_scan(c & ~WARP_PATH, cs);
    if ((threadIdx.x >> 5) == 0) {
      const u32 excl = lookback(a.status, t, cs.tile_agg, epoch, st);
      if ((threadIdx.x & 31) == 0 && t == ntiles - 1) st_volatile(n_out, N + excl + cs.tile_agg);
    }
    __syncthreads();
  }
  __syncthreads();
  for (u32 j = threadIdx.x; j < m; j += BLOCK) {
    if (cs.children[j]) atomicAdd(a.tickets + op + j, cs.children[j]);
    if (cs.anti[j] && a.anti) atomicAdd(a.anti + op + j, (u64)cs.anti[j]);
  }
  grid_barrier(st, gen, grp);
  const u64 n_after = ld_volatile(n_out);
  if (n_after > a.cap) {  // stop before any write; the host grows the rows and runs the class again
    for (u64 r = (u64)grp.bid * BLOCK + threadIdx.x; r < N; r += (u64)grp.nblk * BLOCK) {
      if (!a.cls_mask[r]) continue;
      const u32 slot = a.cls_slot[r];
      if (slot != REC_NONE && ~(u32)__ldcg(a.fam_aux + slot) == (u32)r) {
        a.fam_table[slot] = EMPTY_SLOT;
        a.fam_aux[slot] = 0;
      }
    }
    if (grp.bid == 0 && threadIdx.x == 0) {
      st->halt = op;
      st->need_rows = n_after;
    }
    return 2;
  }
  // C: write
  for (u32 t = grp.bid; t < ntiles; t += grp.nblk) {
    const u64 r = (u64)t * BLOCK + threadIdx.x;
    u32 mine = 0;
    if (r < N && a.cls_mask[r]) {
      const u32 slot = a.cls_slot[r];
      if (slot != REC_NONE && ~(u32)__ldcg(a.fam_aux + slot) == (u32)r) mine = __ldcg(a.cls_children + r);
    }
    const u32 off = block_excl_scan(mine & ~WARP_PATH, cs);
    if (threadIdx.x == 0) {
      const u64 s = ld_volatile(a.status + t);
      cs.tile_excl = (u32)s - cs.tile_agg;  // the look-back left the inclusive prefix
    }
    __syncthreads();
    const u64 base = N + cs.tile_excl;
    class_tile<W, ALG, true>(a, R, cg, N, r, keys, coeffs, cs, base, off, mine);
    __syncthreads();
  }
  return 0;
}
