// sk_opsurf.cu — the interpreter's join, project and aggregate operators on
// packed key columns (the operator surface behind strata_op_join /
// strata_op_project / strata_op_aggregate).
//
// A binary relation column is a packed key (c0 << shift) | c1 (u32 or u64).
//
// join — one binary rule body  h(X,Z) :- a(X,Y), b(Y,Z)  evaluated as the
//   reference's `solve` does it (strata-eval/src/seminaive.rs:215-298: every
//   binding of the body, one per pair of unifying tuples) with the head built
//   as (X, Z) (`build_head`, naive.rs:526) and the annotations multiplied
//   (Ann::otimes, value.rs:56: Bool AND, Trop checked +).  `b` arrives sorted
//   by (Y, Z); its CSR over Y is built on the device and the bindings are
//   enumerated by the same load-balanced expand the fixpoint rounds use.  The
//   output is in a's order and unsorted; sort + dedup / min-merge (the other
//   operators) finish the round.
//
// project — the head built from one body atom's binding: each output column
//   is an input column or a constant (build_head for a single-atom body).
//
// select — `unify` of one atom with a repeated variable or a constant
//   (naive.rs:407-455): the rows whose two columns agree, or whose column
//   equals a constant.
//
// intersect — two atoms over the same two variables: the rows of a also in
//   b (sorted), with the Trop product of both weights.
//
// semijoin — a negated (or existence-only) atom: the rows whose probe key is
//   absent from (present in) a sorted relation.
//
// aggregate — `eval_aggregate_rule` + `fold_aggregate` (naive.rs:300-391):
//   over bindings sorted by key, the group is key >> group_shift; count is
//   the number of bindings of the group, sum / min / max fold an int64
//   aggregand column.  Reduce-then-scan: per-tile group-head counts, one
//   scan, the heads' positions, then one warp per group folds its run.
#include "sk_ops.cuh"
#include "sk_prims.cuh"

namespace sk {
namespace {

constexpr int NT = 256;
constexpr int AG_ITEMS = 8;
constexpr uint32_t AG_TILE = NT * AG_ITEMS;

inline unsigned grid_of(uint64_t n, uint64_t per) { return (unsigned)ceil_div(n ? n : 1, per); }

// The operator surface carries Trop weights as int64 with INT64_MAX = +inf;
// the kernels use codes with +inf = WInf (sk_prims.cuh).  Finite weights
// above WFinMax have no code on this surface.
__global__ void k_op_to_codes(const int64_t* __restrict__ in, uint64_t n, int64_t* __restrict__ out,
                              uint32_t* status) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t v = in[i];
  if (v == INT64_MAX) {
    out[i] = WInf<int64_t>::v;
  } else {
    if (v > WFinMax<int64_t>::v) atomicOr(status, ST_SENTINEL);
    out[i] = v;
  }
}

__global__ void k_op_from_codes(int64_t* w, uint64_t n) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && w[i] == WInf<int64_t>::v) w[i] = INT64_MAX;
}

template <class KI, class KO>
__global__ void k_project(const KI* __restrict__ in, uint64_t n, int in_shift, int sel_hi, int sel_lo,
                          uint64_t const_hi, uint64_t const_lo, int out_shift, KO* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t k = (uint64_t)in[i];
  const uint64_t lowmask = in_shift >= 64 ? ~0ull : ((1ull << in_shift) - 1);
  const uint64_t c0 = in_shift >= 64 ? 0ull : (k >> in_shift), c1 = k & lowmask;
  const uint64_t hi = sel_hi == 0 ? c0 : sel_hi == 1 ? c1 : const_hi;
  const uint64_t lo = sel_lo == 0 ? c0 : sel_lo == 1 ? c1 : const_lo;
  out[i] = sel_hi == 3 ? (KO)lo : (KO)((hi << out_shift) | lo);
}

template <class K>
__device__ __forceinline__ bool ag_head(const K* keys, uint64_t i, int gshift) {
  if (i == 0) return true;
  const uint64_t a = gshift >= 64 ? 0ull : ((uint64_t)keys[i - 1] >> gshift);
  const uint64_t b = gshift >= 64 ? 0ull : ((uint64_t)keys[i] >> gshift);
  return a != b;
}

template <class K>
__global__ void __launch_bounds__(NT) k_ag_count(const K* __restrict__ keys, uint64_t n, int gshift,
                                                 uint64_t* __restrict__ tile_cnt, uint32_t* status) {
  __shared__ uint32_t s_red[NT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * AG_TILE;
  uint32_t c = 0;
  uint32_t flags = 0;
#pragma unroll
  for (int j = 0; j < AG_ITEMS; j++) {
    const uint64_t i = base + (uint64_t)j * NT + tid;
    if (i < n) {
      c += ag_head(keys, i, gshift) ? 1u : 0u;
      if (i > 0 && keys[i - 1] > keys[i]) flags |= ST_BOUNDS;  // the input must be sorted
    }
  }
  c = warp_sum(c);
  if (lane == 0) s_red[warp] = c;
  if (flags) atomicOr(status, flags);
  __syncthreads();
  if (tid == 0) {
    uint64_t t = 0;
    for (int w = 0; w < NT / 32; w++) t += s_red[w];
    tile_cnt[blockIdx.x] = t;
  }
}

// Positions of the group heads, in order: starts[g] = first binding of group g.
template <class K>
__global__ void __launch_bounds__(NT) k_ag_starts(const K* __restrict__ keys, uint64_t n, int gshift,
                                                  const uint64_t* __restrict__ tile_off, uint64_t* __restrict__ starts,
                                                  K* __restrict__ groups) {
  __shared__ uint32_t s_scan[NT / 32 + 1];
  const int tid = threadIdx.x;
  // thread t owns AG_ITEMS consecutive bindings, so heads come out in order
  const uint64_t b = (uint64_t)blockIdx.x * AG_TILE + (uint64_t)tid * AG_ITEMS;
  uint32_t hm = 0;
#pragma unroll
  for (int j = 0; j < AG_ITEMS; j++)
    if (b + j < n && ag_head(keys, b + j, gshift)) hm |= 1u << j;
  uint32_t tot;
  const uint32_t ex = block_excl_sum<NT>((uint32_t)__popc(hm), s_scan, &tot);
  uint64_t at = tile_off[blockIdx.x] + ex;
  for (int j = 0; j < AG_ITEMS; j++) {
    if ((hm >> j) & 1u) {
      starts[at] = b + j;
      groups[at] = gshift >= 64 ? K(0) : (K)((uint64_t)keys[b + j] >> gshift);
      at++;
    }
  }
}

// One warp per group: fold the aggregand over [starts[g], starts[g+1]).
// op: 0 count, 1 sum (wrapping i64), 2 min, 3 max.
__global__ void __launch_bounds__(NT) k_ag_fold(const uint64_t* __restrict__ starts, uint64_t n_groups, uint64_t n,
                                                const int64_t* __restrict__ vals, int op, int64_t* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * (NT / 32);
  for (uint64_t g = ((uint64_t)blockIdx.x * NT + threadIdx.x) >> 5; g < n_groups; g += warps) {
    const uint64_t a = starts[g], e = g + 1 < n_groups ? starts[g + 1] : n;
    if (op == 0) {
      if (lane == 0) out[g] = (int64_t)(e - a);
      continue;
    }
    long long acc = op == 1 ? 0ll : op == 2 ? INT64_MAX : INT64_MIN;
    for (uint64_t i = a + lane; i < e; i += 32) {
      const long long v = vals[i];
      if (op == 1) acc = (long long)((unsigned long long)acc + (unsigned long long)v);
      else if (op == 2) acc = v < acc ? v : acc;
      else acc = v > acc ? v : acc;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const long long t = __shfl_xor_sync(kFull, acc, o);
      if (op == 1) acc = (long long)((unsigned long long)acc + (unsigned long long)t);
      else if (op == 2) acc = t < acc ? t : acc;
      else acc = t > acc ? t : acc;
    }
    if (lane == 0) out[g] = acc;
  }
}

// Row filter + compaction shared by select and intersect: `keep` decides a
// row (and its output weight); per-tile counts, one scan, then the write in
// input order (a thread owns SE_ITEMS consecutive rows).
constexpr int SE_ITEMS = 8;
constexpr uint32_t SE_TILE = NT * SE_ITEMS;

// unify of one atom with a repeated variable or a constant
// (strata-eval/src/naive.rs:407-455): mode 0 keeps c0 == c1, 1 keeps
// c0 == k, 2 keeps c1 == k.
template <class K>
struct SelectRow {
  int shift, mode;
  uint64_t k;
  __device__ bool keep(K key, const int64_t* w, uint64_t i, int64_t* ow, uint32_t*) const {
    const uint64_t x = (uint64_t)key;
    const uint64_t c0 = shift >= 64 ? 0ull : (x >> shift);
    const uint64_t c1 = x & (shift >= 64 ? ~0ull : ((1ull << shift) - 1));
    if (w) *ow = w[i];
    return mode == 0 ? c0 == c1 : mode == 1 ? c0 == k : c1 == k;
  }
};

// a ∩ b on whole keys (two atoms over the same variables): binary search of
// each a key in the sorted b; Trop weight a.w ⊗ b.w on the operator
// surface's codes.
template <class K>
struct IntersectRow {
  const K* b;
  const int64_t* bw;
  uint64_t nb;
  __device__ bool keep(K key, const int64_t* w, uint64_t i, int64_t* ow, uint32_t* flags) const {
    const uint64_t j = lower_bound_dev(b, 0, nb, key);
    if (j >= nb || b[j] != key) return false;
    if (w) {
      const int64_t x = w[i], y = bw[j];
      if (x == INT64_MAX || y == INT64_MAX) {
        *ow = INT64_MAX;
      } else {
        const int64_t xa = x > WFinMax<int64_t>::v ? 0 : x, ya = y > WFinMax<int64_t>::v ? 0 : y;
        if (x > WFinMax<int64_t>::v || y > WFinMax<int64_t>::v) *flags |= ST_SENTINEL;
        *ow = trop_mul(xa, ya, 0, flags);
        if (*ow == WInf<int64_t>::v) *ow = INT64_MAX;
      }
    }
    return true;
  }
};

// Stratified negation / semi-join (negation_holds, naive.rs:537-566): keep
// row i when probe[i] (the row's own key when probe is NULL) is absent from
// (anti) or present in the sorted b; weights pass through unchanged.
template <class K>
struct SemiRow {
  const K* probe;
  const K* b;
  uint64_t nb;
  bool anti;
  __device__ bool keep(K key, const int64_t* w, uint64_t i, int64_t* ow, uint32_t*) const {
    const K pk = probe ? probe[i] : key;
    const uint64_t j = nb ? lower_bound_dev(b, 0, nb, pk) : 0;
    const bool found = j < nb && b[j] == pk;
    if (w) *ow = w[i];
    return anti ? !found : found;
  }
};

template <class K, class P>
__global__ void __launch_bounds__(NT) k_filter_count(const K* __restrict__ keys, const int64_t* __restrict__ w,
                                                     uint64_t n, P pred, uint64_t* __restrict__ tile_cnt,
                                                     uint32_t* status) {
  __shared__ uint32_t s_red[NT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t b = (uint64_t)blockIdx.x * SE_TILE + (uint64_t)tid * SE_ITEMS;
  uint32_t c = 0, flags = 0;
  for (int j = 0; j < SE_ITEMS; j++) {
    int64_t ow;
    if (b + j < n && pred.keep(keys[b + j], w, b + j, &ow, &flags)) c++;
  }
  c = warp_sum(c);
  if (lane == 0) s_red[warp] = c;
  if (flags) atomicOr(status, flags);
  __syncthreads();
  if (tid == 0) {
    uint64_t t = 0;
    for (int q = 0; q < NT / 32; q++) t += s_red[q];
    tile_cnt[blockIdx.x] = t;
  }
}

template <class K, class P>
__global__ void __launch_bounds__(NT) k_filter_write(const K* __restrict__ keys, const int64_t* __restrict__ w,
                                                     uint64_t n, P pred, const uint64_t* __restrict__ tile_off,
                                                     K* __restrict__ out, int64_t* __restrict__ out_w,
                                                     uint32_t* status) {
  __shared__ uint32_t s_scan[NT / 32 + 1];
  const int tid = threadIdx.x;
  const uint64_t b = (uint64_t)blockIdx.x * SE_TILE + (uint64_t)tid * SE_ITEMS;
  uint32_t km = 0, flags = 0;
  int64_t ws[SE_ITEMS];
#pragma unroll
  for (int j = 0; j < SE_ITEMS; j++) {
    ws[j] = 0;
    if (b + j < n && pred.keep(keys[b + j], w, b + j, &ws[j], &flags)) km |= 1u << j;
  }
  uint32_t tot;
  const uint32_t ex = block_excl_sum<NT>((uint32_t)__popc(km), s_scan, &tot);
  uint64_t at = tile_off[blockIdx.x] + ex;
#pragma unroll
  for (int j = 0; j < SE_ITEMS; j++) {
    if ((km >> j) & 1u) {
      out[at] = keys[b + j];
      if (w) out_w[at] = ws[j];
      at++;
    }
  }
  if (flags) atomicOr(status, flags);
}

template <class K, class P>
uint64_t filter_rows(strata_ctx* ctx, const K* keys, const int64_t* w, uint64_t n, const P& pred, K* out,
                     int64_t* out_w) {
  if (n == 0) return 0;
  const uint64_t tiles = ceil_div(n, SE_TILE);
  DBuf<uint64_t> toff(ctx, tiles + 1);
  k_filter_count<K, P><<<(unsigned)tiles, NT, 0, ctx->stream>>>(keys, w, n, pred, toff.p, ctx->d_status);
  after_launch(ctx, "k_filter_count");
  scan_tile_sums(ctx, toff.p, tiles);
  k_filter_write<K, P><<<(unsigned)tiles, NT, 0, ctx->stream>>>(keys, w, n, pred, toff.p, out, out_w, ctx->d_status);
  after_launch(ctx, "k_filter_write");
  uint64_t r;
  read_u64(ctx, toff.p + tiles, &r, 1);
  sync_and_check(ctx);
  return r;
}

}  // namespace

template <class K>
uint64_t op_join(strata_ctx* ctx, const K* dk, const int64_t* dw, uint64_t nd, int d_shift, const K* rk,
                 const int64_t* rw, uint64_t nr, int r_shift, int out_shift, K* out, int64_t* out_w, uint64_t out_cap,
                 bool* written) {
  *written = false;
  if (nd == 0 || nr == 0) {
    *written = out != nullptr;
    return 0;
  }
  const bool trop = dw != nullptr;
  K last;
  SK_CUDA(cudaMemcpyAsync(&last, rk + (nr - 1), sizeof(K), cudaMemcpyDeviceToHost, ctx->stream));
  SK_CUDA(cudaStreamSynchronize(ctx->stream));
  const uint64_t n_nodes = (r_shift >= (int)(8 * sizeof(K)) ? 0ull : ((uint64_t)last >> r_shift)) + 1;
  if (n_nodes > (1ull << 32)) fail(STRATA_E_UNSUPPORTED, "join column values must be below 2^32");
  DBuf<uint32_t> off(ctx, n_nodes + 1), nbr(ctx, nr + 1);
  build_csr<K>(ctx, rk, nr, r_shift, n_nodes, off.p, nbr.p);
  DBuf<uint64_t> pos(ctx, nd + 1);
  const uint64_t dmask = d_shift >= 64 ? ~0ull : ((1ull << d_shift) - 1);
  expand_offsets<K>(ctx, dk, nd, 0, dmask, off.p, n_nodes, pos.p);
  uint64_t T = 0;
  read_u64(ctx, pos.p + nd, &T, 1);
  sync_and_check(ctx);  // an unsorted `b` shows up here as a bounds status
  if (!out || out_cap < T) return T;
  *written = true;
  if (T == 0) return 0;
  ctx->wshift = 0;
  if (trop) {
    DBuf<int64_t> cd(ctx, nd), cr(ctx, nr);
    k_op_to_codes<<<grid_of(nd, NT), NT, 0, ctx->stream>>>(dw, nd, cd.p, ctx->d_status);
    after_launch(ctx, "k_op_to_codes");
    k_op_to_codes<<<grid_of(nr, NT), NT, 0, ctx->stream>>>(rw, nr, cr.p, ctx->d_status);
    after_launch(ctx, "k_op_to_codes");
    expand_emit<K, int64_t, true>(ctx, dk, cd.p, nd, pos.p, T, 0, dmask, d_shift, ~0ull, out_shift, 0, off.p, n_nodes,
                                  nbr.p, nr, cr.p, out, out_w);
    k_op_from_codes<<<grid_of(T, NT), NT, 0, ctx->stream>>>(out_w, T);
    after_launch(ctx, "k_op_from_codes");
  } else {
    expand_emit<K, int32_t, false>(ctx, dk, nullptr, nd, pos.p, T, 0, dmask, d_shift, ~0ull, out_shift, 0, off.p,
                                   n_nodes, nbr.p, nr, nullptr, out, nullptr);
  }
  sync_and_check(ctx);
  return T;
}

template <class KI, class KO>
void op_project(strata_ctx* ctx, const KI* in, uint64_t n, int in_shift, int sel_hi, int sel_lo, uint64_t const_hi,
                uint64_t const_lo, int out_shift, KO* out) {
  if (n == 0) return;
  k_project<KI, KO><<<grid_of(n, NT), NT, 0, ctx->stream>>>(in, n, in_shift, sel_hi, sel_lo, const_hi, const_lo,
                                                           out_shift, out);
  after_launch(ctx, "k_project");
  sync_and_check(ctx);
}

template <class K>
uint64_t op_aggregate(strata_ctx* ctx, const K* keys, const int64_t* vals, uint64_t n, int gshift, int op, K* groups,
                      int64_t* out_vals) {
  if (n == 0) return 0;
  const uint64_t tiles = ceil_div(n, AG_TILE);
  DBuf<uint64_t> toff(ctx, tiles + 1);
  k_ag_count<K><<<(unsigned)tiles, NT, 0, ctx->stream>>>(keys, n, gshift, toff.p, ctx->d_status);
  after_launch(ctx, "k_ag_count");
  scan_tile_sums(ctx, toff.p, tiles);
  uint64_t ng = 0;
  read_u64(ctx, toff.p + tiles, &ng, 1);
  sync_and_check(ctx);  // unsorted input: STRATA_E_CUDA with the bounds message before anything is written
  DBuf<uint64_t> starts(ctx, ng + 1);
  k_ag_starts<K><<<(unsigned)tiles, NT, 0, ctx->stream>>>(keys, n, gshift, toff.p, starts.p, groups);
  after_launch(ctx, "k_ag_starts");
  const unsigned g = (unsigned)std::min<uint64_t>(ceil_div(ng, NT / 32), (uint64_t)ctx->num_sms * 16);
  k_ag_fold<<<g ? g : 1, NT, 0, ctx->stream>>>(starts.p, ng, n, vals, op, out_vals);
  after_launch(ctx, "k_ag_fold");
  sync_and_check(ctx);
  return ng;
}

template <class K>
uint64_t op_select(strata_ctx* ctx, const K* keys, const int64_t* w, uint64_t n, int shift, int mode, uint64_t k,
                   K* out, int64_t* out_w) {
  return filter_rows<K, SelectRow<K>>(ctx, keys, w, n, SelectRow<K>{shift, mode, k}, out, out_w);
}

template <class K>
uint64_t op_intersect(strata_ctx* ctx, const K* a, const int64_t* aw, uint64_t na, const K* b, const int64_t* bw,
                      uint64_t nb, K* out, int64_t* out_w) {
  if (nb == 0) return 0;
  return filter_rows<K, IntersectRow<K>>(ctx, a, aw, na, IntersectRow<K>{b, bw, nb}, out, out_w);
}

template <class K>
uint64_t op_semijoin(strata_ctx* ctx, const K* rows, const int64_t* w, uint64_t n, const K* probe, const K* b,
                     uint64_t nb, bool anti, K* out, int64_t* out_w) {
  return filter_rows<K, SemiRow<K>>(ctx, rows, w, n, SemiRow<K>{probe, b, nb, anti}, out, out_w);
}

template uint64_t op_semijoin<uint32_t>(strata_ctx*, const uint32_t*, const int64_t*, uint64_t, const uint32_t*,
                                        const uint32_t*, uint64_t, bool, uint32_t*, int64_t*);
template uint64_t op_semijoin<uint64_t>(strata_ctx*, const uint64_t*, const int64_t*, uint64_t, const uint64_t*,
                                        const uint64_t*, uint64_t, bool, uint64_t*, int64_t*);
template uint64_t op_select<uint32_t>(strata_ctx*, const uint32_t*, const int64_t*, uint64_t, int, int, uint64_t,
                                      uint32_t*, int64_t*);
template uint64_t op_select<uint64_t>(strata_ctx*, const uint64_t*, const int64_t*, uint64_t, int, int, uint64_t,
                                      uint64_t*, int64_t*);
template uint64_t op_intersect<uint32_t>(strata_ctx*, const uint32_t*, const int64_t*, uint64_t, const uint32_t*,
                                         const int64_t*, uint64_t, uint32_t*, int64_t*);
template uint64_t op_intersect<uint64_t>(strata_ctx*, const uint64_t*, const int64_t*, uint64_t, const uint64_t*,
                                         const int64_t*, uint64_t, uint64_t*, int64_t*);
template uint64_t op_join<uint32_t>(strata_ctx*, const uint32_t*, const int64_t*, uint64_t, int, const uint32_t*,
                                    const int64_t*, uint64_t, int, int, uint32_t*, int64_t*, uint64_t, bool*);
template uint64_t op_join<uint64_t>(strata_ctx*, const uint64_t*, const int64_t*, uint64_t, int, const uint64_t*,
                                    const int64_t*, uint64_t, int, int, uint64_t*, int64_t*, uint64_t, bool*);
template void op_project<uint32_t, uint32_t>(strata_ctx*, const uint32_t*, uint64_t, int, int, int, uint64_t, uint64_t,
                                             int, uint32_t*);
template void op_project<uint32_t, uint64_t>(strata_ctx*, const uint32_t*, uint64_t, int, int, int, uint64_t, uint64_t,
                                             int, uint64_t*);
template void op_project<uint64_t, uint32_t>(strata_ctx*, const uint64_t*, uint64_t, int, int, int, uint64_t, uint64_t,
                                             int, uint32_t*);
template void op_project<uint64_t, uint64_t>(strata_ctx*, const uint64_t*, uint64_t, int, int, int, uint64_t, uint64_t,
                                             int, uint64_t*);
template uint64_t op_aggregate<uint32_t>(strata_ctx*, const uint32_t*, const int64_t*, uint64_t, int, int, uint32_t*,
                                         int64_t*);
template uint64_t op_aggregate<uint64_t>(strata_ctx*, const uint64_t*, const int64_t*, uint64_t, int, int, uint64_t*,
                                         int64_t*);

}  // namespace sk
