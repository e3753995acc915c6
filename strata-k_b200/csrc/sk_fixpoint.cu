// sk_fixpoint.cu — device-resident semi-naive drivers for the linear rule
// shapes of the hot path.
//
// Semantics follow strata-eval/src/seminaive.rs:
//   * a bootstrap full step seeds Δ with every derived tuple (:90);
//   * each delta round evaluates the recursive rule once with the recursive
//     atom ranging over Δ (:142-170), ⊕-combines the derivations into the
//     relation and takes Δ' = the changed tuples with their merged value
//     (:183-208; Relation::combine, store.rs:34-48);
//   * a Trop stratum that is still changing after `universe + 2` delta rounds
//     is a negative-weight cycle (:92-103), where `universe` is the number of
//     distinct symbols in the EDB (naive.rs:143-155);
//   * Trop ⊗ is checked i64 addition with +inf absorption (strata-ir/src/trop.rs:52-62).
//
// One round on the device: expand (Δ ⋈ CSR) -> radix sort -> run reduction ->
// merge-path merge/diff against the full relation.  The host reads two
// scalars per round (the expand size and the new |Δ|) plus the status word.
#include "sk_ops.cuh"
#include "sk_prims.cuh"
#include "sk_rel.cuh"

#include <cmath>
#include <type_traits>

namespace sk {
namespace {

template <class W> struct SortVal;
template <> struct SortVal<int32_t> { using type = uint32_t; };
template <> struct SortVal<int64_t> { using type = uint64_t; };

template <class K, class W>
struct Rel {
  DBuf<K> k;
  DBuf<W> w;
  uint64_t n = 0;
  void reserve(uint64_t m, bool trop) {
    k.reserve_grow(m);
    if (trop) w.reserve_grow(m);
  }
  void swap(Rel& o) {
    k.swap(o.k);
    w.swap(o.w);
    std::swap(n, o.n);
  }
};

template <class W>
struct Csr {
  DBuf<uint32_t> off;
  DBuf<uint32_t> nbr;
  DBuf<W> w;
  uint64_t n_nodes = 0;
  uint64_t m = 0;
};

struct JoinSpec {
  int jshift;
  uint64_t jmask;
  int pshift;
  uint64_t pmask;
  int out_pshift;
  int out_vshift;
};

inline uint64_t low_mask(int bits) { return bits >= 64 ? ~0ull : ((1ull << bits) - 1); }

// Per-round scratch, reused across rounds (grown geometrically).
template <class K, class W>
struct Scratch {
  DBuf<uint64_t> pos;
  DBuf<K> ck, ck2, uk;
  DBuf<W> cw, cw2, uw;
  DBuf<uint64_t> counts;
  explicit Scratch(strata_ctx* ctx) {
    pos.ctx = ck.ctx = ck2.ctx = uk.ctx = ctx;
    cw.ctx = cw2.ctx = uw.ctx = ctx;
    counts.ctx = ctx;
    counts.reserve(4);
  }
};

struct Acct {  // per-phase accounting for strata_fix_stats
  double sort_ms = 0, join_ms = 0, diff_ms = 0, merge_ms = 0, setup_ms = 0, finish_ms = 0;
  int setup_t = -1;
  uint64_t sort_b = 0, join_b = 0, diff_b = 0, merge_b = 0;
  uint32_t sort_l = 0, join_l = 0, diff_l = 0, merge_l = 0;
  uint64_t cands = 0;
};

// Read count values and the status word with one synchronization.
inline void read_checked(strata_ctx* ctx, const uint64_t* d, uint64_t* out, int count) {
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, d, sizeof(uint64_t) * count, cudaMemcpyDeviceToHost,
                          ctx->stream));
  sync_and_check(ctx);
  std::memcpy(out, ctx->h_scalar, sizeof(uint64_t) * count);
}

// C = reduce(sort(expand(Δ ⋈ csr))): the distinct derived keys of one round
// (Trop: min weight each), left in s.uk / s.uw.  Returns |C|.
template <class K, class W, bool TROP>
uint64_t derive(strata_ctx* ctx, const K* dk, const W* dw, uint64_t nd, const Csr<W>& csr,
                const JoinSpec& js, int key_bits, Scratch<K, W>& s, PhaseTimer& pt, Acct& a) {
  using V = typename SortVal<W>::type;
  if (nd == 0) return 0;
  const uint64_t l0 = ctx->launches;
  int t = pt.begin(&a.join_ms);
  s.pos.reserve_grow(nd + 1);
  expand_offsets<K>(ctx, dk, nd, js.jshift, js.jmask, csr.off.p, csr.n_nodes, s.pos.p);
  uint64_t T = 0;
  read_checked(ctx, s.pos.p + nd, &T, 1);
  if (T == 0) {
    pt.end(t);
    a.join_l += (uint32_t)(ctx->launches - l0);
    return 0;
  }
  if (T > kMaxSortN)
    fail(STRATA_E_UNSUPPORTED, "one round derives " + std::to_string(T) +
                                   " candidates; the per-round limit is 2^30-1");
  s.ck.reserve_grow(T);
  s.ck2.reserve_grow(T);
  if (TROP) {
    s.cw.reserve_grow(T);
    s.cw2.reserve_grow(T);
  }
  expand_emit<K, W, TROP>(ctx, dk, dw, nd, s.pos.p, T, js.jshift, js.jmask, js.pshift, js.pmask,
                          js.out_pshift, js.out_vshift, csr.off.p, csr.n_nodes, csr.nbr.p, csr.m,
                          TROP ? csr.w.p : nullptr, s.ck.p, TROP ? s.cw.p : nullptr);
  pt.end(t);
  const uint64_t ksz = sizeof(K), wsz = TROP ? sizeof(W) : 0;
  a.join_b += nd * (ksz + wsz + 8) + T * (4 + wsz) + T * (ksz + wsz);
  a.join_l += (uint32_t)(ctx->launches - l0);
  a.cands += T;

  const uint64_t l1 = ctx->launches;
  t = pt.begin(&a.sort_ms);
  K* kp = s.ck.p;
  K* ka = s.ck2.p;
  V* vp = reinterpret_cast<V*>(s.cw.p);
  V* va = reinterpret_cast<V*>(s.cw2.p);
  radix_sort<K, V>(ctx, &kp, &ka, &vp, &va, TROP, T, key_bits, false);
  pt.end(t);
  a.sort_b += 2 * T * (ksz + wsz) * (uint64_t)((key_bits + 7) / 8);
  a.sort_l += (uint32_t)(ctx->launches - l1);

  const uint64_t l2 = ctx->launches;
  t = pt.begin(&a.diff_ms);
  s.uk.reserve_grow(T);
  if (TROP) s.uw.reserve_grow(T);
  reduce_runs<K, W, TROP>(ctx, kp, reinterpret_cast<W*>(vp), T, s.uk.p, TROP ? s.uw.p : nullptr,
                          s.counts.p);
  uint64_t nu = 0;
  read_u64(ctx, s.counts.p, &nu, 1);
  kprof_add_last(ctx, K_REDUCE_RUNS, nu * (ksz + wsz));
  pt.end(t);
  a.diff_b += T * (ksz + wsz) + nu * (ksz + wsz);
  a.diff_l += (uint32_t)(ctx->launches - l2);
  return nu;
}

// Semi-naive loop: full/delta are sorted unique; runs until Δ is empty.
template <class K, class W, bool TROP>
void fix_loop(strata_ctx* ctx, Rel<K, W>& full, Rel<K, W>& delta, const Csr<W>& csr,
              const JoinSpec& js, int key_bits, uint64_t cap, Scratch<K, W>& s, PhaseTimer& pt,
              Acct& a, uint64_t* rounds_out) {
  Rel<K, W> full2, dnext;
  full2.k.ctx = full2.w.ctx = dnext.k.ctx = dnext.w.ctx = ctx;
  uint64_t rounds = 0;
  const uint64_t ksz = sizeof(K), wsz = TROP ? sizeof(W) : 0;
  while (delta.n > 0) {
    rounds++;
    const uint64_t nu = derive<K, W, TROP>(ctx, delta.k.p, TROP ? delta.w.p : nullptr, delta.n, csr,
                                           js, key_bits, s, pt, a);
    if (nu == 0) {
      delta.n = 0;
    } else {
      const uint64_t l0 = ctx->launches;
      const int t = pt.begin(&a.merge_ms);
      full2.reserve(full.n + nu, TROP);
      dnext.reserve(nu, TROP);
      merge_diff<K, W, TROP>(ctx, full.k.p, TROP ? full.w.p : nullptr, full.n, s.uk.p,
                             TROP ? s.uw.p : nullptr, nu, full2.k.p, TROP ? full2.w.p : nullptr,
                             dnext.k.p, TROP ? dnext.w.p : nullptr, s.counts.p);
      uint64_t c[2];
      read_checked(ctx, s.counts.p, c, 2);
      kprof_add_last(ctx, K_MERGE_DIFF, (c[0] + c[1]) * (ksz + wsz));
      pt.end(t);
      a.merge_b += (full.n + nu) * (ksz + wsz) + (c[0] + c[1]) * (ksz + wsz);
      a.merge_l += (uint32_t)(ctx->launches - l0);
      full.swap(full2);
      full.n = c[0];
      delta.swap(dnext);
      delta.n = c[1];
    }
    // The interpreter checks the cap after every delta round, including the
    // one that finds no change (seminaive.rs:99-103).
    if (TROP && cap && rounds > cap)
      fail(STRATA_E_NEG_CYCLE, "negative-weight cycle: tropical stratum diverges");
  }
  *rounds_out = rounds;
}

// Sort + reduce a packed relation in place into `out` (unique, Trop min).
template <class K, class W, bool TROP>
void normalize(strata_ctx* ctx, DBuf<K>& keys, DBuf<W>& w, uint64_t n, int key_bits, Rel<K, W>& out) {
  using V = typename SortVal<W>::type;
  DBuf<K> ka(ctx, n + 1);
  DBuf<W> wa;
  wa.ctx = ctx;
  if (TROP) wa.reserve(n + 1);
  K* kp = keys.p;
  K* kalt = ka.p;
  V* vp = reinterpret_cast<V*>(w.p);
  V* valt = reinterpret_cast<V*>(wa.p);
  radix_sort<K, V>(ctx, &kp, &kalt, &vp, &valt, TROP, n, key_bits, true);
  out.reserve(n + 1, TROP);
  DBuf<uint64_t> cnt(ctx, 1);
  reduce_runs<K, W, TROP>(ctx, kp, reinterpret_cast<W*>(vp), n, out.k.p, TROP ? out.w.p : nullptr, cnt.p);
  read_u64(ctx, cnt.p, &out.n, 1);
}

// CSR of an edge relation keyed by `join_col` (0 = src, 1 = dst) with the
// other column as neighbour; Trop weights min-merged per (join, nbr).
template <class KC, class W, bool TROP>
void build_edge_csr(strata_ctx* ctx, const EdgeCols& e, int join_col, int jbits, int vbits,
                    uint64_t n_nodes, Csr<W>& csr) {
  DBuf<KC> keys(ctx, e.n + 1);
  DBuf<W> w;
  w.ctx = ctx;
  if (TROP) w.reserve(e.n + 1);
  const uint32_t* c0 = join_col == 0 ? e.src : e.dst;
  const uint32_t* c1 = join_col == 0 ? e.dst : e.src;
  pack_pairs<KC, W, TROP>(ctx, c0, c1, e.w, e.inf, e.n, vbits, keys.p, TROP ? w.p : nullptr);
  Rel<KC, W> r;
  r.k.ctx = r.w.ctx = ctx;
  normalize<KC, W, TROP>(ctx, keys, w, e.n, jbits + vbits, r);
  csr.off.ctx = csr.nbr.ctx = csr.w.ctx = ctx;
  csr.off.reserve(n_nodes + 1);
  csr.nbr.reserve(r.n + 1);
  build_csr<KC>(ctx, r.k.p, r.n, vbits, n_nodes, csr.off.p, csr.nbr.p);
  if (TROP) csr.w = std::move(r.w);
  csr.n_nodes = n_nodes;
  csr.m = r.n;
}

template <class K, class W, bool TROP>
strata_rel* finish_rel(strata_ctx* ctx, Rel<K, W>& full, int shift) {
  strata_rel* rel = new strata_rel();
  rel->trop = TROP;
  rel->key_bytes = sizeof(K);
  rel->w_bytes = TROP ? sizeof(W) : 0;
  rel->shift = shift;
  rel->wshift = TROP ? ctx->wshift : 0;
  rel->n = full.n;
  rel->keys = full.k.detach();
  rel->w = TROP ? (void*)full.w.detach() : nullptr;
  return rel;
}

struct EventTimer {
  strata_ctx* ctx;
  cudaEvent_t a = nullptr, b = nullptr;
  explicit EventTimer(strata_ctx* c) : ctx(c) {
    SK_CUDA(cudaEventCreate(&a));
    SK_CUDA(cudaEventCreate(&b));
    SK_CUDA(cudaEventRecord(a, ctx->stream));
  }
  double stop() {
    SK_CUDA(cudaEventRecord(b, ctx->stream));
    SK_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    SK_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
  }
  ~EventTimer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

void fill_stats(strata_fix_stats* st, const Acct& a, uint64_t rounds, uint64_t result,
                uint64_t universe, int key_bits, int wbytes, double ms, uint64_t launches) {
  if (!st) return;
  st->rounds = rounds;
  st->candidates = a.cands;
  st->result_tuples = result;
  st->universe = universe;
  st->key_bits = key_bits;
  st->weight_bytes = wbytes;
  st->device_ms = ms;
  st->sort_ms = a.sort_ms;
  st->join_ms = a.join_ms;
  st->diff_ms = a.diff_ms;
  st->merge_ms = a.merge_ms;
  st->sort_bytes = a.sort_b;
  st->join_bytes = a.join_b;
  st->diff_bytes = a.diff_b;
  st->merge_bytes = a.merge_b;
  st->sort_launches = a.sort_l;
  st->join_launches = a.join_l;
  st->diff_launches = a.diff_l;
  st->merge_launches = a.merge_l;
  const uint64_t phase = (uint64_t)a.sort_l + a.join_l + a.diff_l + a.merge_l;
  st->other_launches = (uint32_t)(launches > phase ? launches - phase : 0);
  st->setup_ms = a.setup_ms;
  st->finish_ms = a.finish_ms;
}

// ---- direct-addressed plan ---------------------------------------------------------
// Index over (c0, c1) in [0, n0) × [0, n1): a membership bitmap (Bool), an
// int32 weight array (Trop), the marks of the current Δ and, for Trop, the
// snapshot of Δ's weights that the next round reads.
template <class W>
struct DenseIdx {
  DBuf<uint32_t> bits;   // Bool membership
  DBuf<uint32_t> marks;  // Δ: the entries the last round marked
  DBuf<W> D;             // Trop weight codes (WAbs<W> = absent)
  DBuf<W> Dprev;         // Trop: Δ's weights as the round that made it left them
  DBuf<uint32_t> hidx, hseg, hmask;  // heads (key-head row or marks word, CSR segment, member mask)
  DBuf<uint8_t> hg;                  // key-head group sizes
  DBuf<uint64_t> hpos, hsums;        // head degree prefix; per-tile sums of the head compaction
  DenseLayout lay{};
  uint64_t entries = 0;
  uint64_t words() const { return entries / 32; }
};

// Bytes the index needs (D and Dprev at `wbytes` per entry for Trop, the
// bitmap for Bool, the marks); the plan is used when they stay within budget.
inline double dense_bytes(bool trop, int wbytes, uint64_t n0, uint64_t n1) {
  const double rows = (double)n1, width = (double)((n0 + 31) & ~31ull);  // the wider of the two layouts
  const double rows2 = (double)n0, width2 = (double)((n1 + 31) & ~31ull);
  const double e = std::max(rows * width, rows2 * width2);
  return (trop ? 2.0 * wbytes * e : e / 8.0) + e / 8.0;
}
constexpr double kDenseBudget = 16e9;

inline bool want_dense(strata_ctx* ctx, bool trop, bool narrow, uint64_t n0, uint64_t n1) {
  const long double e = (long double)n0 * (long double)n1;
  const bool fits = e < 9.0e18L && n0 < (1ull << 32) && n1 < (1ull << 32) &&
                    dense_bytes(trop, narrow ? 4 : 8, n0, n1) <= kDenseBudget;
  if (ctx->plan == 3) fail(STRATA_E_UNSUPPORTED, "the bit-row plan applies to Bool transitive closure only");
  if (ctx->plan == 1) return false;
  if (ctx->plan == 2 && !fits) fail(STRATA_E_UNSUPPORTED, "the direct-addressed plan needs an index within 16 GB");
  return fits;
}

// `colmajor`: the next round joins on c1 (rows by c1), else on c0.
template <bool TROP, class W>
void dense_alloc(strata_ctx* ctx, DenseIdx<W>& X, uint64_t n0, uint64_t n1, int b1, bool colmajor) {
  X.bits.ctx = X.D.ctx = X.Dprev.ctx = X.marks.ctx = ctx;
  X.hidx.ctx = X.hseg.ctx = X.hmask.ctx = X.hg.ctx = X.hpos.ctx = X.hsums.ctx = ctx;
  X.lay = dense_layout(b1, n0, n1, colmajor);
  X.entries = X.lay.entries;
  if (!TROP) {
    X.bits.reserve(X.words() + 1);
    SK_CUDA(cudaMemsetAsync(X.bits.p, 0, (X.words() + 1) * 4, ctx->stream));
  }
  X.marks.reserve(X.words() + 1);
  SK_CUDA(cudaMemsetAsync(X.marks.p, 0, (X.words() + 1) * 4, ctx->stream));
  X.hsums.reserve(dense_word_heads_sums(X.lay));
  if (TROP) {
    X.D.reserve(X.entries + 1);
    X.Dprev.reserve(X.entries + 1);
  }
}

// A round whose Δ is a key list (the bootstrap src ⋈ edge): key heads, then
// the expand, which marks the new / improved entries (the next Δ).  Returns
// the candidate count (a bound on the marks set).
template <class K, bool TROP, class W>
uint64_t dense_round_keys(strata_ctx* ctx, const K* dk, const W* dw, uint64_t nd, const Csr<W>& csr,
                          const JoinSpec& js, DenseIdx<W>& X, DBuf<uint64_t>& splits, PhaseTimer& pt, Acct& a) {
  if (nd == 0) return 0;
  const uint64_t l0 = ctx->launches;
  const int t = pt.begin(&a.join_ms);
  X.hpos.reserve_grow(nd + 1);
  X.hidx.reserve_grow(nd + 1);
  X.hseg.reserve_grow(nd + 1);
  X.hg.reserve_grow(nd + 1);
  DBuf<uint64_t> sums(ctx, dense_heads_sums(nd));
  uint64_t h3[3];
  dense_heads<K>(ctx, dk, nd, js.jshift, js.jmask, csr.off.p, csr.n_nodes, sums.p, X.hidx.p, X.hpos.p, X.hseg.p,
                 X.hg.p, h3);
  const uint64_t nh = h3[0], T = h3[1], cands = h3[2];  // heads; (group, edge) outputs; candidates
  if (T) {
    splits.reserve_grow(ceil_div(nh + T, dense_tile_size()) + 2);
    dense_expand<K, TROP, W>(ctx, dk, dw, nd, X.hidx.p, X.hpos.p, X.hseg.p, X.hg.p, nh, T, cands, js.pshift, js.pmask,
                          js.out_pshift, js.out_vshift, csr.nbr.p, csr.m, TROP ? csr.w.p : nullptr, X.lay,
                          TROP ? nullptr : X.bits.p, TROP ? X.D.p : nullptr, X.marks.p, splits.p);
  }
  pt.end(t);
  const uint64_t wsz = TROP ? sizeof(W) : 0;
  a.join_b += nd * (sizeof(K) + wsz) + nh * 17 + T * (4 + wsz) + cands * (TROP ? sizeof(W) : 4);
  a.join_l += (uint32_t)(ctx->launches - l0);
  a.cands += cands;
  return cands;
}

// Semi-naive rounds with Δ in the marks: word heads (which clear the marks
// and snapshot Δ's weights), then the expand marks Δ'.  A round runs while
// Δ is non-empty; `bound` is an upper bound on the entries marked now.
template <bool TROP, class W>
void fix_loop_dense(strata_ctx* ctx, const Csr<W>& csr, const JoinSpec& js, DenseIdx<W>& X, uint64_t bound,
                    uint64_t cap, PhaseTimer& pt, Acct& a, uint64_t* rounds_out) {
  DBuf<uint64_t> splits;
  splits.ctx = ctx;
  uint64_t rounds = 0;
  for (;;) {
    const uint64_t l0 = ctx->launches;
    const int t = pt.begin(&a.join_ms);
    const uint64_t hcap = std::min<uint64_t>(X.words(), bound) + 1;
    X.hidx.reserve_grow(hcap);
    X.hmask.reserve_grow(hcap);
    X.hseg.reserve_grow(hcap);
    X.hpos.reserve_grow(hcap);
    uint64_t h4[4];
    dense_word_heads<TROP, W>(ctx, X.marks.p, X.lay, csr.off.p, csr.n_nodes, X.hsums.p, X.hidx.p, X.hmask.p,
                           X.hpos.p, X.hseg.p, TROP ? X.D.p : nullptr, TROP ? X.Dprev.p : nullptr, h4);
    const uint64_t nh = h4[0], T = h4[1], cands = h4[2], nd = h4[3];
    if (nd == 0) {
      pt.end(t);
      a.join_b += X.words() * 4;
      a.join_l += (uint32_t)(ctx->launches - l0);
      break;
    }
    rounds++;
    if (T) {
      splits.reserve_grow(ceil_div(nh + T, dense_tile_size()) + 2);
      dense_expand_words<TROP, W>(ctx, X.hidx.p, X.hmask.p, X.hpos.p, X.hseg.p, nh, T, cands, nd,
                               TROP ? X.Dprev.p : nullptr, js.out_pshift, js.out_vshift, csr.nbr.p, csr.m,
                               TROP ? csr.w.p : nullptr, X.lay, TROP ? nullptr : X.bits.p, TROP ? X.D.p : nullptr,
                               X.marks.p, splits.p);
    }
    pt.end(t);
    const uint64_t wsz = TROP ? sizeof(W) : 0;
    // marks read and cleared, head records written and read, Δ weights
    // snapshot (read, write, read), edges, probes
    a.join_b += X.words() * 4 * 2 + nh * 20 * 2 + nd * 3 * wsz + T * (4 + wsz) + cands * (TROP ? sizeof(W) : 4);
    a.join_l += (uint32_t)(ctx->launches - l0);
    a.cands += cands;
    bound = std::min<uint64_t>(cands, X.entries);
    if (TROP && cap && rounds > cap)
      fail(STRATA_E_NEG_CYCLE, "negative-weight cycle: tropical stratum diverges");
  }
  *rounds_out = rounds;
}

// Compact the index into a sorted relation.
template <class K, bool TROP, class W>
void dense_finish(strata_ctx* ctx, DenseIdx<W>& X, int b1, Rel<K, W>& full, uint64_t upper) {
  (void)b1;
  const uint64_t cap = std::min<uint64_t>(upper, X.lay.n0 * X.lay.n1) + 1;
  full.reserve(cap, TROP);
  full.n = dense_compact<K, TROP, W>(ctx, X.bits.p, TROP ? X.D.p : nullptr, X.lay, full.k.p,
                                     TROP ? full.w.p : nullptr, cap);
}

// ---- TC-shaped drivers: head(X,Z) :- edge(X,Y), head(Y,Z) -----------------------
template <class K, class W, bool TROP>
strata_rel* run_tc_shape(strata_ctx* ctx, const EdgeCols& e, int b0, int b1, int bsrc,
                         uint64_t n_nodes_dst, uint64_t universe, uint64_t cap, strata_fix_stats* st,
                         EventTimer& et, uint64_t l_start, uint64_t n_nodes_src, bool dense) {
  PhaseTimer pt(ctx);
  Acct a;
  a.setup_t = pt.begin(&a.setup_ms);
  uint32_t plan = 1;
  const int key_bits = b0 + b1;
  // path0 = normalize(edge): every edge is derived by the base rule.
  Rel<K, W> full, delta;
  full.k.ctx = full.w.ctx = delta.k.ctx = delta.w.ctx = ctx;
  {
    DBuf<K> keys(ctx, e.n + 1);
    DBuf<W> w;
    w.ctx = ctx;
    if (TROP) w.reserve(e.n + 1);
    pack_pairs<K, W, TROP>(ctx, e.src, e.dst, e.w, e.inf, e.n, b1, keys.p, TROP ? w.p : nullptr);
    normalize<K, W, TROP>(ctx, keys, w, e.n, key_bits, full);
  }
  // In-CSR: Y -> X (join on the edge's dst), key bits b1 + bsrc.
  Csr<W> csr;
  if (b1 + bsrc <= 32)
    build_edge_csr<uint32_t, W, TROP>(ctx, e, 1, b1, bsrc, n_nodes_dst, csr);
  else
    build_edge_csr<uint64_t, W, TROP>(ctx, e, 1, b1, bsrc, n_nodes_dst, csr);
  delta.reserve(full.n + 1, TROP);
  delta.n = full.n;
  SK_CUDA(cudaMemcpyAsync(delta.k.p, full.k.p, full.n * sizeof(K), cudaMemcpyDeviceToDevice, ctx->stream));
  if (TROP)
    SK_CUDA(cudaMemcpyAsync(delta.w.p, full.w.p, full.n * sizeof(W), cudaMemcpyDeviceToDevice, ctx->stream));
  // Δ(Y,Z): join value Y = key >> b1, kept Z = key & mask(b1), out = (X << b1) | Z.
  JoinSpec js{b1, low_mask(b0), 0, low_mask(b1), 0, b1};
  Scratch<K, W> s(ctx);
  uint64_t rounds = 0;
  if (dense) {
    plan = 2;
    DenseIdx<W> X;
    // Δ(Y,Z) joins on c0: row-major index.
    dense_alloc<TROP, W>(ctx, X, n_nodes_src, n_nodes_dst, b1, false);
    // the seed is also the first Δ: its entries are marked
    if (TROP) dense_seed<K, true, W>(ctx, full.k.p, full.w.p, full.n, X.lay, X.bits.p, X.D.p, X.marks.p);
    else dense_seed<K, false, W>(ctx, full.k.p, nullptr, full.n, X.lay, X.bits.p, nullptr, X.marks.p);
    pt.end(a.setup_t);
    fix_loop_dense<TROP, W>(ctx, csr, js, X, full.n, cap, pt, a, &rounds);
    const int tf = pt.begin(&a.finish_ms);
    dense_finish<K, TROP, W>(ctx, X, b1, full, X.entries);
    pt.end(tf);
  }
  if (plan == 1) {
    pt.end(a.setup_t);
    fix_loop<K, W, TROP>(ctx, full, delta, csr, js, key_bits, cap, s, pt, a, &rounds);
  }
  const double ms = et.stop();
  pt.collect();
  kprof_collect(ctx);
  fill_stats(st, a, rounds, full.n, universe, key_bits, TROP ? sizeof(W) : 0, ms, ctx->launches - l_start);
  if (st) st->plan = plan;
  return finish_rel<K, W, TROP>(ctx, full, b1);
}

struct Layout {
  int b0, b1, bsrc;
  uint64_t n_nodes;      // max dst + 1
  uint64_t n_nodes_src;  // max src + 1
  bool wide_key;
};

Layout tc_layout(strata_ctx* ctx, const EdgeCols& e) {
  const uint32_t ms = max_u32(ctx, e.src, e.n), md = max_u32(ctx, e.dst, e.n);
  Layout L;
  L.b0 = std::max(1, bits_for(ms));
  L.b1 = std::max(1, bits_for(md));
  L.bsrc = L.b0;
  L.n_nodes = (uint64_t)md + 1;
  L.n_nodes_src = (uint64_t)ms + 1;
  L.wide_key = L.b0 + L.b1 > 32;
  return L;
}

// Weight code shift of a wide (int64) fixpoint.  Every value the schedule
// forms within the round cap is one seed weight plus at most cap + 2 edge
// weights (or cap + 3 edge weights for the edge-seeded shape); [lo, hi]
// bounds all of them.  Codes are value - s with finite codes up to
// INT64_MAX - 2 (sk_prims.cuh), so s = max(0, hi - (INT64_MAX - 2)) in
// {0, 1, 2} keeps every value up to i64::MAX representable (a sum beyond it
// is the reference's overflow error, detected on codes), and lo must still
// have a code: lo >= INT64_MIN + s, else STRATA_E_WEIGHT_RANGE.
int64_t wide_shift(strata_ctx* ctx, const int64_t* ew, const uint8_t* einf, uint64_t ne, const int64_t* sw,
                   const uint8_t* sinf, uint64_t ns, uint64_t cap) {
  int64_t emn = 0, emx = 0, smn = 0, smx = 0;
  if (!weight_range(ctx, ew, einf, ne, &emn, &emx)) emn = emx = 0;
  if (ns && !weight_range(ctx, sw, sinf, ns, &smn, &smx)) smn = smx = 0;
  const __int128 L = (__int128)cap + 3;
  const __int128 kMax = INT64_MAX, kMin = INT64_MIN;
  __int128 hi = (__int128)std::max<int64_t>(smx, 0) + L * (__int128)std::max<int64_t>(emx, 0);
  __int128 lo = (__int128)std::min<int64_t>(smn, 0) + L * (__int128)std::min<int64_t>(emn, 0);
  if (hi > kMax) hi = kMax;
  if (lo < kMin) lo = kMin;
  const __int128 fin = kMax - 2;
  const int64_t s = hi > fin ? (int64_t)(hi - fin) : 0;
  if (lo < kMin + s)
    fail(STRATA_E_WEIGHT_RANGE,
         "finite tropical weights span nearly all of i64 (sums within the round cap can reach both i64::MIN and "
         "i64::MAX): no 64-bit code keeps them apart from +inf");
  return s;
}

// Narrow (int32) Trop weights are exact when every derived sum within the
// round cap stays inside int32: at most (cap + 2) edges plus one seed weight.
bool narrow_ok(uint64_t universe, uint64_t max_edge_w, uint64_t max_seed_w) {
  const long double bound =
      (long double)(universe + 4) * (long double)max_edge_w + (long double)max_seed_w;
  return bound < 2147483000.0L;
}

// Bool closure on bit rows (sk_bitset.cu); the result is compacted from the
// final bit rows in (X, Z) order.
template <class K>
strata_rel* run_tc_bitset(strata_ctx* ctx, const EdgeCols& e, const Layout& L, strata_fix_stats* st, EventTimer& et,
                          uint64_t l_start) {
  Acct a;
  Rel<K, int32_t> full;
  full.k.ctx = full.w.ctx = ctx;
  uint64_t rounds = 0, round_bytes = 0;
  full.n = tc_bool_bitset<K>(ctx, e.src, e.dst, e.n, L.n_nodes_src, L.n_nodes, L.b1, full.k, &rounds, &round_bytes);
  a.join_b = round_bytes;
  const double ms = et.stop();
  kprof_collect(ctx);
  fill_stats(st, a, rounds, full.n, 0, L.b0 + L.b1, 0, ms, ctx->launches - l_start);
  if (st) {
    st->plan = 3;
    st->join_ms = ms;
  }
  return finish_rel<K, int32_t, false>(ctx, full, L.b1);
}

}  // namespace

strata_rel* fix_tc_bool(strata_ctx* ctx, const EdgeCols& e, strata_fix_stats* st) {
  if (st) std::memset(st, 0, sizeof(*st));
  reset_status(ctx);
  const uint64_t l_start = ctx->launches;
  ctx->wshift = 0;
  EventTimer et(ctx);
  if (e.n == 0) {
    strata_rel* rel = new strata_rel();
    return rel;
  }
  const Layout L = tc_layout(ctx, e);
  if (ctx->plan == 3 || ctx->plan == 0) {
    const bool fits = tc_bool_bitset_fits(ctx, L.n_nodes_src, L.n_nodes, e.n);
    if (ctx->plan == 3 && !fits) fail(STRATA_E_UNSUPPORTED, "the bit-row plan needs its bit matrices within 8 GB");
    if (fits) {
      if (!L.wide_key) return run_tc_bitset<uint32_t>(ctx, e, L, st, et, l_start);
      return run_tc_bitset<uint64_t>(ctx, e, L, st, et, l_start);
    }
  }
  const bool dense = want_dense(ctx, false, true, L.n_nodes_src, L.n_nodes);
  if (!L.wide_key)
    return run_tc_shape<uint32_t, int32_t, false>(ctx, e, L.b0, L.b1, L.bsrc, L.n_nodes, 0, 0, st, et, l_start,
                                                  L.n_nodes_src, dense);
  return run_tc_shape<uint64_t, int32_t, false>(ctx, e, L.b0, L.b1, L.bsrc, L.n_nodes, 0, 0, st, et, l_start,
                                                L.n_nodes_src, dense);
}

strata_rel* fix_trop_paths(strata_ctx* ctx, const EdgeCols& e, strata_fix_stats* st) {
  if (st) std::memset(st, 0, sizeof(*st));
  reset_status(ctx);
  const uint64_t l_start = ctx->launches;
  ctx->wshift = 0;
  EventTimer et(ctx);
  if (e.n == 0) {
    strata_rel* rel = new strata_rel();
    rel->trop = true;
    rel->w_bytes = 8;
    return rel;
  }
  const Layout L = tc_layout(ctx, e);
  const uint64_t limit = (uint64_t)std::max(max_u32(ctx, e.src, e.n), (uint32_t)(L.n_nodes - 1)) + 1;
  const uint64_t universe = count_distinct_ids(ctx, e.src, e.n, e.dst, e.n, nullptr, 0, limit);
  const uint64_t cap = universe + 2;
  const bool narrow = !ctx->force_wide && narrow_ok(universe, max_abs_weight(ctx, e.w, e.inf, e.n), 0);
  ctx->wshift = narrow ? 0 : wide_shift(ctx, e.w, e.inf, e.n, nullptr, nullptr, 0, cap);
  const bool dense = want_dense(ctx, true, narrow, L.n_nodes_src, L.n_nodes);
  const uint64_t ns = L.n_nodes_src;
  if (!L.wide_key) {
    if (narrow)
      return run_tc_shape<uint32_t, int32_t, true>(ctx, e, L.b0, L.b1, L.bsrc, L.n_nodes, universe, cap, st, et,
                                                   l_start, ns, dense);
    return run_tc_shape<uint32_t, int64_t, true>(ctx, e, L.b0, L.b1, L.bsrc, L.n_nodes, universe, cap, st, et,
                                                 l_start, ns, dense);
  }
  if (narrow)
    return run_tc_shape<uint64_t, int32_t, true>(ctx, e, L.b0, L.b1, L.bsrc, L.n_nodes, universe, cap, st, et,
                                                 l_start, ns, dense);
  return run_tc_shape<uint64_t, int64_t, true>(ctx, e, L.b0, L.b1, L.bsrc, L.n_nodes, universe, cap, st, et,
                                               l_start, ns, dense);
}

// ---- MSSP: dist(S,Y) :- src(S), edge(S,Y). dist(S,Z) :- dist(S,Y), edge(Y,Z). ----
namespace {

template <class K, class W>
strata_rel* run_mssp(strata_ctx* ctx, const uint32_t* sources, const int64_t* src_w,
                     const uint8_t* src_inf, uint64_t ns, const EdgeCols& e, int b0, int b1,
                     int besrc, uint64_t n_nodes_src, uint64_t universe, uint64_t cap,
                     strata_fix_stats* st, EventTimer& et, uint64_t l_start, uint64_t n0, uint64_t n1,
                     bool dense) {
  PhaseTimer pt(ctx);
  Acct a;
  a.setup_t = pt.begin(&a.setup_ms);
  const int key_bits = b0 + b1;
  // src as a unary Trop relation keyed by S (min over duplicate facts).
  Rel<K, W> srcu;
  srcu.k.ctx = srcu.w.ctx = ctx;
  {
    DBuf<K> keys(ctx, ns + 1);
    DBuf<W> w(ctx, ns + 1);
    pack_pairs<K, W, true>(ctx, nullptr, sources, src_w, src_inf, ns, 0, keys.p, w.p);
    normalize<K, W, true>(ctx, keys, w, ns, b0, srcu);
  }
  // Out-CSR: Y -> Z with weights (join on the edge's src), key bits besrc + b1.
  Csr<W> csr;
  if (besrc + b1 <= 32)
    build_edge_csr<uint32_t, W, true>(ctx, e, 0, besrc, b1, n_nodes_src, csr);
  else
    build_edge_csr<uint64_t, W, true>(ctx, e, 0, besrc, b1, n_nodes_src, csr);
  Scratch<K, W> s(ctx);
  const JoinSpec boot{0, ~0ull, 0, ~0ull, b1, 0};
  // Δ(S,Y): join Y = key & mask(b1), kept S = key >> b1, out = (S << b1) | Z.
  const JoinSpec step{0, low_mask(b1), b1, low_mask(b0), b1, 0};
  if (dense) {
    DenseIdx<W> X;
    // Δ(S,Y) joins on c1: column-major index, so Δ' comes out sorted by Y.
    dense_alloc<true, W>(ctx, X, n0, n1, b1, true);
    dense_seed<K, true, W>(ctx, nullptr, nullptr, 0, X.lay, X.bits.p, X.D.p, nullptr);
    Rel<K, W> full;
    full.k.ctx = full.w.ctx = ctx;
    DBuf<uint64_t> splits;
    splits.ctx = ctx;
    pt.end(a.setup_t);
    // Bootstrap: every derivation of src ⋈ edge, all new; its marks are
    // the first Δ.
    const uint64_t bound = dense_round_keys<K, true, W>(ctx, srcu.k.p, srcu.w.p, srcu.n, csr, boot, X, splits, pt, a);
    uint64_t rounds = 0;
    fix_loop_dense<true, W>(ctx, csr, step, X, std::min<uint64_t>(bound, X.entries), cap, pt, a, &rounds);
    const int tf = pt.begin(&a.finish_ms);
    dense_finish<K, true, W>(ctx, X, b1, full, X.entries);
    pt.end(tf);
    const double ms = et.stop();
    pt.collect();
    kprof_collect(ctx);
    fill_stats(st, a, rounds, full.n, universe, key_bits, sizeof(W), ms, ctx->launches - l_start);
    if (st) st->plan = 2;
    return finish_rel<K, W, true>(ctx, full, b1);
  }
  pt.end(a.setup_t);
  // Bootstrap: dist0 = min-reduce(src ⋈ edge), all of it new.
  const uint64_t nb = derive<K, W, true>(ctx, srcu.k.p, srcu.w.p, srcu.n, csr, boot, key_bits, s, pt, a);
  Rel<K, W> full, delta;
  full.k.ctx = full.w.ctx = delta.k.ctx = delta.w.ctx = ctx;
  full.reserve(nb + 1, true);
  delta.reserve(nb + 1, true);
  full.n = delta.n = nb;
  if (nb) {
    SK_CUDA(cudaMemcpyAsync(full.k.p, s.uk.p, nb * sizeof(K), cudaMemcpyDeviceToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(full.w.p, s.uw.p, nb * sizeof(W), cudaMemcpyDeviceToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(delta.k.p, s.uk.p, nb * sizeof(K), cudaMemcpyDeviceToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(delta.w.p, s.uw.p, nb * sizeof(W), cudaMemcpyDeviceToDevice, ctx->stream));
  }
  uint64_t rounds = 0;
  fix_loop<K, W, true>(ctx, full, delta, csr, step, key_bits, cap, s, pt, a, &rounds);
  const double ms = et.stop();
  pt.collect();
  kprof_collect(ctx);
  fill_stats(st, a, rounds, full.n, universe, key_bits, sizeof(W), ms, ctx->launches - l_start);
  if (st) st->plan = 1;
  return finish_rel<K, W, true>(ctx, full, b1);
}

}  // namespace

strata_rel* fix_mssp(strata_ctx* ctx, const uint32_t* sources, const int64_t* src_w,
                     const uint8_t* src_inf, uint64_t ns, const EdgeCols& e, strata_fix_stats* st) {
  if (st) std::memset(st, 0, sizeof(*st));
  reset_status(ctx);
  const uint64_t l_start = ctx->launches;
  ctx->wshift = 0;
  EventTimer et(ctx);
  if (ns == 0 || e.n == 0) {
    strata_rel* rel = new strata_rel();
    rel->trop = true;
    rel->w_bytes = 8;
    if (st) {
      st->universe = 0;
    }
    return rel;
  }
  const uint32_t mS = max_u32(ctx, sources, ns);
  const uint32_t mes = max_u32(ctx, e.src, e.n), med = max_u32(ctx, e.dst, e.n);
  const int b0 = std::max(1, bits_for(mS));
  const int b1 = std::max(1, bits_for(med));
  const int besrc = std::max(1, bits_for(mes));
  const uint64_t limit = (uint64_t)std::max(mS, std::max(mes, med)) + 1;
  const uint64_t universe = count_distinct_ids(ctx, sources, ns, e.src, e.n, e.dst, e.n, limit);
  const uint64_t cap = universe + 2;
  const bool narrow = !ctx->force_wide && narrow_ok(universe, max_abs_weight(ctx, e.w, e.inf, e.n),
                                                    max_abs_weight(ctx, src_w, src_inf, ns));
  ctx->wshift = narrow ? 0 : wide_shift(ctx, e.w, e.inf, e.n, src_w, src_inf, ns, cap);
  const uint64_t nn = (uint64_t)mes + 1;
  const uint64_t n0 = (uint64_t)mS + 1, n1 = (uint64_t)med + 1;
  const bool dense = want_dense(ctx, true, narrow, n0, n1);
  if (b0 + b1 <= 32) {
    if (narrow)
      return run_mssp<uint32_t, int32_t>(ctx, sources, src_w, src_inf, ns, e, b0, b1, besrc, nn, universe, cap, st,
                                         et, l_start, n0, n1, dense);
    return run_mssp<uint32_t, int64_t>(ctx, sources, src_w, src_inf, ns, e, b0, b1, besrc, nn, universe, cap, st,
                                       et, l_start, n0, n1, dense);
  }
  if (narrow)
    return run_mssp<uint64_t, int32_t>(ctx, sources, src_w, src_inf, ns, e, b0, b1, besrc, nn, universe, cap, st, et,
                                       l_start, n0, n1, dense);
  return run_mssp<uint64_t, int64_t>(ctx, sources, src_w, src_inf, ns, e, b0, b1, besrc, nn, universe, cap, st, et,
                                     l_start, n0, n1, dense);
}

// ---- relation handles ---------------------------------------------------------------

void rel_to_host(strata_ctx* ctx, const strata_rel* rel, uint32_t* src, uint32_t* dst, int64_t* w,
                 uint8_t* inf) {
  const uint64_t n = rel->n;
  ctx->wshift = rel->wshift;  // the codes of this relation decode with its own shift
  if (n == 0) return;
  DBuf<uint32_t> c0(ctx, n), c1(ctx, n);
  DBuf<int64_t> ow;
  DBuf<uint8_t> oi;
  ow.ctx = oi.ctx = ctx;
  const bool want_w = rel->trop && (w || inf);
  if (want_w) {
    ow.reserve(n);
    oi.reserve(n);
  }
  if (rel->key_bytes == 4) {
    const uint32_t* k = static_cast<const uint32_t*>(rel->keys);
    if (!rel->trop) unpack_pairs<uint32_t, int32_t, false>(ctx, k, nullptr, n, rel->shift, c0.p, c1.p, nullptr, nullptr);
    else if (rel->w_bytes == 4) unpack_pairs<uint32_t, int32_t, true>(ctx, k, (const int32_t*)rel->w, n, rel->shift, c0.p, c1.p, want_w ? ow.p : nullptr, want_w ? oi.p : nullptr);
    else unpack_pairs<uint32_t, int64_t, true>(ctx, k, (const int64_t*)rel->w, n, rel->shift, c0.p, c1.p, want_w ? ow.p : nullptr, want_w ? oi.p : nullptr);
  } else {
    const uint64_t* k = static_cast<const uint64_t*>(rel->keys);
    if (!rel->trop) unpack_pairs<uint64_t, int32_t, false>(ctx, k, nullptr, n, rel->shift, c0.p, c1.p, nullptr, nullptr);
    else if (rel->w_bytes == 4) unpack_pairs<uint64_t, int32_t, true>(ctx, k, (const int32_t*)rel->w, n, rel->shift, c0.p, c1.p, want_w ? ow.p : nullptr, want_w ? oi.p : nullptr);
    else unpack_pairs<uint64_t, int64_t, true>(ctx, k, (const int64_t*)rel->w, n, rel->shift, c0.p, c1.p, want_w ? ow.p : nullptr, want_w ? oi.p : nullptr);
  }
  if (src) SK_CUDA(cudaMemcpyAsync(src, c0.p, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (dst) SK_CUDA(cudaMemcpyAsync(dst, c1.p, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (want_w && w) SK_CUDA(cudaMemcpyAsync(w, ow.p, n * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (want_w && inf) SK_CUDA(cudaMemcpyAsync(inf, oi.p, n, cudaMemcpyDeviceToHost, ctx->stream));
  sync_and_check(ctx);
}

uint64_t rel_fingerprint(strata_ctx* ctx, const strata_rel* rel) {
  if (rel->n == 0) return 0;
  ctx->wshift = rel->wshift;
  if (rel->key_bytes == 4) {
    const uint32_t* k = static_cast<const uint32_t*>(rel->keys);
    if (!rel->trop) return fingerprint<uint32_t, int32_t, false>(ctx, k, nullptr, rel->n, rel->shift);
    if (rel->w_bytes == 4) return fingerprint<uint32_t, int32_t, true>(ctx, k, (const int32_t*)rel->w, rel->n, rel->shift);
    return fingerprint<uint32_t, int64_t, true>(ctx, k, (const int64_t*)rel->w, rel->n, rel->shift);
  }
  const uint64_t* k = static_cast<const uint64_t*>(rel->keys);
  if (!rel->trop) return fingerprint<uint64_t, int32_t, false>(ctx, k, nullptr, rel->n, rel->shift);
  if (rel->w_bytes == 4) return fingerprint<uint64_t, int32_t, true>(ctx, k, (const int32_t*)rel->w, rel->n, rel->shift);
  return fingerprint<uint64_t, int64_t, true>(ctx, k, (const int64_t*)rel->w, rel->n, rel->shift);
}

void rel_free(strata_ctx* ctx, strata_rel* rel) {
  if (!rel) return;
  if (ctx) {
    dev_free(ctx, rel->keys);
    dev_free(ctx, rel->w);
  }
  delete rel;
}

}  // namespace sk
