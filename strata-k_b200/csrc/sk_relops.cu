// sk_relops.cu — the interpreter's operator surface on sorted packed keys.
//
//   expand_offsets + expand_emit : scan/join/project of Δ against a CSR index
//       of the EDB relation on the join column (replaces bj_count/bj_emit,
//       strata-gpu/src/sort.rs:115-145, and bjt_emit :176; the reference
//       copies the counts to the host for a prefix sum, tc.rs:67-78).
//   reduce_runs : dedup (Bool ⊕ = OR) or min-by-key (Trop ⊕ = min) of sorted
//       candidates (flag_unique/scatter_unique, sort.rs:69-111; sort_min_dev
//       :465-513).
//   merge_diff  : full ∪ C and Δ' = C ∖ full (Bool) or C's new-or-improved
//       rows (Trop) in ONE merge-path pass (diff_flag :146, diff_improve :192,
//       and the concat + full re-sort of tc.rs:124-144 / trop.rs:177-213).
//   build_csr, pack/unpack, distinct-id count, fingerprint : plumbing.
//
// Every kernel is single-pass over its inputs; cross-tile offsets come from
// the bounded decoupled look-back in sk_prims.cuh.
#include "sk_ops.cuh"
#include "sk_prims.cuh"

namespace sk {
namespace {

constexpr int NT = 256;

// ---------------------------------------------------------------------------
// expand: offsets
// ---------------------------------------------------------------------------
constexpr int EO_ITEMS = 16;
constexpr uint32_t EO_TILE = NT * EO_ITEMS;

template <class K>
__global__ void __launch_bounds__(NT)
    k_expand_offsets(const K* __restrict__ dkeys, uint64_t n, int jshift, uint64_t jmask,
                     const uint32_t* __restrict__ off, uint64_t n_nodes, uint64_t* __restrict__ pos,
                     uint64_t* states, uint32_t* counter, uint32_t* status, uint32_t gmax,
                     unsigned long long* cand_total) {
  __shared__ uint32_t s_tile;
  __shared__ uint64_t s_warp[NT / 32 + 1];
  __shared__ uint64_t s_excl;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t tile = claim_tile(counter, &s_tile);
  const uint64_t wbase = (uint64_t)tile * EO_TILE + (uint64_t)warp * 32 * EO_ITEMS;
  uint64_t vals[EO_ITEMS];
  uint64_t carry = 0;
  unsigned long long cands = 0;
#pragma unroll
  for (int j = 0; j < EO_ITEMS; j++) {
    const uint64_t idx = wbase + j * 32 + lane;
    uint64_t deg = 0;
    if (idx < n) {
      const uint64_t jv = ((uint64_t)dkeys[idx] >> jshift) & jmask;
      if (jv < n_nodes) deg = (uint64_t)(off[jv + 1] - off[jv]);
      cands += deg;
      // grouped: a follower of a run (same join value, same gmax block) has no outputs
      if (gmax && idx % gmax != 0 && (((uint64_t)dkeys[idx - 1] >> jshift) & jmask) == jv) deg = 0;
    }
    const uint64_t incl = warp_incl_sum(deg);
    vals[j] = carry + incl - deg;
    carry += __shfl_sync(kFull, incl, 31);
  }
  if (lane == 0) s_warp[warp] = carry;
  if (cand_total) {
    cands = warp_sum(cands);
    if (lane == 0 && cands) atomicAdd(cand_total, cands);
  }
  __syncthreads();
  if (warp == 0) {
    uint64_t w = (lane < NT / 32) ? s_warp[lane] : 0;
    uint64_t wi = warp_incl_sum(w);
    if (lane < NT / 32) s_warp[lane] = wi - w;
    const uint64_t agg = __shfl_sync(kFull, wi, NT / 32 - 1);
    const uint64_t ex = warp_lookback(states, tile, agg, status);
    if (lane == 0) {
      s_excl = ex;
      if (tile == gridDim.x - 1) pos[n] = ex + agg;
    }
  }
  __syncthreads();
  const uint64_t base = s_excl + s_warp[warp];
#pragma unroll
  for (int j = 0; j < EO_ITEMS; j++) {
    const uint64_t idx = wbase + j * 32 + lane;
    if (idx < n) pos[idx] = base + vals[j];
  }
}

// ---------------------------------------------------------------------------
// reduce-then-scan variant of the offsets (no waiting between tiles): one
// kernel sums each tile's degrees, one block scans the tile sums, a third
// kernel writes pos[].  Used where tiles carry little work, so that a
// look-back chain would dominate.
// ---------------------------------------------------------------------------
template <class K>
__device__ __forceinline__ uint64_t group_degree(const K* dkeys, uint64_t idx, int jshift, uint64_t jmask,
                                                 const uint32_t* off, uint64_t n_nodes, uint32_t gmax,
                                                 uint64_t* full_deg) {
  const uint64_t jv = ((uint64_t)dkeys[idx] >> jshift) & jmask;
  uint64_t deg = jv < n_nodes ? (uint64_t)(off[jv + 1] - off[jv]) : 0;
  *full_deg = deg;
  if (gmax && idx % gmax != 0 && (((uint64_t)dkeys[idx - 1] >> jshift) & jmask) == jv) deg = 0;
  return deg;
}

template <class K>
__global__ void __launch_bounds__(NT)
    k_deg_count(const K* __restrict__ dkeys, uint64_t n, int jshift, uint64_t jmask,
                const uint32_t* __restrict__ off, uint64_t n_nodes, uint32_t gmax, uint64_t* __restrict__ tile_sums,
                unsigned long long* cand_total) {
  __shared__ uint64_t s_red[NT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * EO_TILE;
  uint64_t sum = 0;
  unsigned long long cands = 0;
  for (int j = 0; j < EO_ITEMS; j++) {
    const uint64_t idx = base + (uint64_t)j * NT + tid;
    if (idx < n) {
      uint64_t fd;
      sum += group_degree(dkeys, idx, jshift, jmask, off, n_nodes, gmax, &fd);
      cands += fd;
    }
  }
  sum = warp_sum(sum);
  if (cand_total) {
    cands = warp_sum(cands);
    if (lane == 0 && cands) atomicAdd(cand_total, cands);
  }
  if (lane == 0) s_red[warp] = sum;
  __syncthreads();
  if (tid == 0) {
    uint64_t t = 0;
    for (int w = 0; w < NT / 32; w++) t += s_red[w];
    tile_sums[blockIdx.x] = t;
  }
}

// In-place exclusive scan of `count` tile sums in one block; sums[count] = total.
// One block per array; array b starts at sums + b * (count + 1).
__global__ void __launch_bounds__(1024) k_scan_tile_sums(uint64_t* sums, uint64_t count) {
  __shared__ uint64_t s_scratch[1024 / 32 + 1];
  sums += (uint64_t)blockIdx.x * (count + 1);
  const uint64_t per = (count + 1023) / 1024;
  const uint64_t b = (uint64_t)threadIdx.x * per;
  uint64_t local = 0;
  for (uint64_t i = b; i < b + per && i < count; i++) local += sums[i];
  uint64_t tot;
  uint64_t run = block_excl_sum<1024>(local, s_scratch, &tot);
  for (uint64_t i = b; i < b + per && i < count; i++) {
    const uint64_t v = sums[i];
    sums[i] = run;
    run += v;
  }
  if (threadIdx.x == 0) sums[count] = tot;
}

template <class K>
__global__ void __launch_bounds__(NT)
    k_deg_write(const K* __restrict__ dkeys, uint64_t n, int jshift, uint64_t jmask, const uint32_t* __restrict__ off,
                uint64_t n_nodes, uint32_t gmax, const uint64_t* __restrict__ tile_sums, uint64_t n_tiles,
                uint64_t* __restrict__ pos) {
  __shared__ uint64_t s_warp[NT / 32 + 1];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // warp-striped so each warp's 32 x ITEMS items are contiguous (as in the count)
  const uint64_t base = (uint64_t)blockIdx.x * EO_TILE;
  uint64_t vals[EO_ITEMS];
  uint64_t carry = 0;
  const uint64_t wbase = base + (uint64_t)warp * 32 * EO_ITEMS;
#pragma unroll
  for (int j = 0; j < EO_ITEMS; j++) {
    const uint64_t idx = wbase + j * 32 + lane;
    uint64_t deg = 0, fd;
    if (idx < n) deg = group_degree(dkeys, idx, jshift, jmask, off, n_nodes, gmax, &fd);
    const uint64_t incl = warp_incl_sum(deg);
    vals[j] = carry + incl - deg;
    carry += __shfl_sync(kFull, incl, 31);
  }
  if (lane == 0) s_warp[warp] = carry;
  __syncthreads();
  if (warp == 0) {
    uint64_t w = (lane < NT / 32) ? s_warp[lane] : 0;
    uint64_t wi = warp_incl_sum(w);
    if (lane < NT / 32) s_warp[lane] = wi - w;
  }
  __syncthreads();
  const uint64_t b0 = tile_sums[blockIdx.x] + s_warp[warp];
#pragma unroll
  for (int j = 0; j < EO_ITEMS; j++) {
    const uint64_t idx = wbase + j * 32 + lane;
    if (idx < n) pos[idx] = b0 + vals[j];
  }
  if (blockIdx.x == gridDim.x - 1 && tid == 0) pos[n] = tile_sums[n_tiles];
}

// ---------------------------------------------------------------------------
// expand: load-balanced emit (merge path over item events and outputs)
// ---------------------------------------------------------------------------
constexpr int EE_ITEMS = 6;
constexpr uint32_t EE_TILE = NT * EE_ITEMS;

// #items i with i + pos[i] < d  (i + pos[i] is strictly increasing).
__device__ __forceinline__ uint64_t mp_items_before(const uint64_t* pos, uint64_t n, uint64_t d) {
  uint64_t lo = 0, hi = d < n ? d : n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (mid + pos[mid] < d) lo = mid + 1; else hi = mid;
  }
  return lo;
}

template <class K, class W, bool TROP>
__global__ void __launch_bounds__(NT)
    k_expand_emit(const K* __restrict__ dkeys, const W* __restrict__ dw, uint64_t n,
                  const uint64_t* __restrict__ pos, uint64_t total, int jshift, uint64_t jmask,
                  int pshift, uint64_t pmask, int out_pshift, int out_vshift,
                  const uint32_t* __restrict__ off, uint64_t n_nodes, const uint32_t* __restrict__ nbr,
                  uint64_t n_nbr, const W* __restrict__ nbr_w, K* __restrict__ out, W* __restrict__ out_w,
                  int64_t wshift, uint32_t* status) {
  __shared__ uint64_t s_pos[EE_TILE + 1];
  __shared__ uint32_t s_seg[EE_TILE + 1];
  __shared__ K s_kept[EE_TILE + 1];
  __shared__ W s_w[TROP ? EE_TILE + 1 : 1];
  __shared__ uint64_t s_r[4];
  const int tid = threadIdx.x;
  const uint64_t L = n + total;
  const uint64_t d0 = (uint64_t)blockIdx.x * EE_TILE;
  const uint64_t d1 = d0 + EE_TILE < L ? d0 + EE_TILE : L;
  if (tid == 0) {
    const uint64_t i0 = mp_items_before(pos, n, d0);
    const uint64_t i1 = mp_items_before(pos, n, d1);
    s_r[0] = i0 > 0 ? i0 - 1 : 0;  // first item that may own an output here
    s_r[1] = i1;
    s_r[2] = d0 - i0;              // first output of the tile
    s_r[3] = d1 - i1;              // one past the last output
  }
  __syncthreads();
  const uint64_t a = s_r[0], i1 = s_r[1], o0 = s_r[2], o1 = s_r[3];
  if (i1 - a > EE_TILE + 1) {  // cannot happen for a valid pos[]; never index past smem
    if (tid == 0) atomicOr(status, ST_BOUNDS);
    return;
  }
  const uint32_t cnt = (uint32_t)(i1 - a);  // <= EE_TILE + 1
  for (uint32_t k = tid; k < cnt; k += NT) {
    const uint64_t i = a + k;
    const K key = dkeys[i];
    const uint64_t jv = ((uint64_t)key >> jshift) & jmask;
    s_pos[k] = pos[i];
    s_seg[k] = jv < n_nodes ? off[jv] : 0u;
    s_kept[k] = (K)(((uint64_t)key >> pshift) & pmask);
    if constexpr (TROP) s_w[k] = dw[i];
  }
  __syncthreads();
  uint32_t flags = 0;
  const uint64_t o_end = o1 < total ? o1 : total;  // o1 <= total for a valid pos[]
  for (uint64_t o = o0 + tid; o < o_end; o += NT) {
    // owner = last loaded item with pos <= o
    uint32_t lo = 0, hi = cnt;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (s_pos[mid] <= o) lo = mid + 1; else hi = mid;
    }
    if (lo == 0) { flags |= ST_BOUNDS; continue; }
    const uint32_t li = lo - 1;
    const uint64_t e = (uint64_t)s_seg[li] + (o - s_pos[li]);
    if (e >= n_nbr) { flags |= ST_BOUNDS; continue; }
    const uint32_t v = nbr[e];
    out[o] = (K)(((K)s_kept[li] << out_pshift) | ((K)v << out_vshift));
    if constexpr (TROP) out_w[o] = trop_mul(s_w[li], nbr_w[e], wshift, &flags);
  }
  if (flags) atomicOr(status, flags);
}

// ---------------------------------------------------------------------------
// reduce_runs: one row per distinct key (Trop: minimum weight)
// ---------------------------------------------------------------------------
// Items per thread: odd (conflict-free blocked shared-memory reads); fewer for
// 8-byte rows so the four staging arrays stay within 48 KB.
template <class K, class W, bool TROP>
struct RRCfg {
  static constexpr int ITEMS = (sizeof(K) + (TROP ? sizeof(W) : 0)) > 8 ? 5 : 9;
  static constexpr uint32_t TILE = NT * ITEMS;
};

template <class W>
struct SegMin {  // segmented-min scan state: has a run start, min since it
  bool h;
  W m;
};
template <class W>
__device__ __forceinline__ SegMin<W> seg_combine(SegMin<W> a, SegMin<W> b) {
  SegMin<W> r;
  r.h = a.h | b.h;
  r.m = b.h ? b.m : (a.m < b.m ? a.m : b.m);
  return r;
}

// Run reduction over fixed tiles, reduce-then-scan (no tile waits on
// another, so a run of any length costs no more than its items):
//   k_rr_heads   run heads per tile (key differs from its predecessor);
//   scan         exclusive head counts = the output rank of each tile's first run;
//   k_rr_span    (Trop) the output slot of every run crossing a tile boundary
//                starts at the absent code;
//   k_reduce_runs  each tile stages its heads' keys and the minima of the runs
//                it holds whole, writes them coalesced at its rank, and merges
//                the part of a boundary-crossing run it holds with atomicMin.
__device__ __forceinline__ void atomic_min_w(int32_t* p, int32_t v) { atomicMin(p, v); }
__device__ __forceinline__ void atomic_min_w(int64_t* p, int64_t v) {
  atomicMin(reinterpret_cast<long long*>(p), (long long)v);
}

template <class K, int ITEMS>
__global__ void __launch_bounds__(NT) k_rr_heads(const K* __restrict__ keys, uint64_t n,
                                                 uint64_t* __restrict__ tile_heads) {
  __shared__ uint32_t s_red[NT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t t0 = (uint64_t)blockIdx.x * (NT * ITEMS);
  uint32_t c = 0;
#pragma unroll
  for (int q = 0; q < ITEMS; q++) {
    const uint64_t i = t0 + (uint64_t)q * NT + tid;
    if (i < n) c += (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
  }
  c = warp_sum(c);
  if (lane == 0) s_red[warp] = c;
  __syncthreads();
  if (tid == 0) {
    uint32_t t = 0;
#pragma unroll
    for (int w = 0; w < NT / 32; w++) t += s_red[w];
    tile_heads[blockIdx.x] = t;
  }
}

template <class K, class W>
__global__ void k_rr_span(const K* __restrict__ keys, uint64_t n, uint32_t tile_len, uint64_t tiles,
                          const uint64_t* __restrict__ rank0, W* __restrict__ out_w) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x + 1;  // boundary before tile t
  if (t >= tiles) return;
  const uint64_t p = t * tile_len;
  if (p < n && keys[p] == keys[p - 1]) out_w[rank0[t] - 1] = WAbs<W>::v;
}

template <class K, class W, bool TROP>
__global__ void __launch_bounds__(NT)
    k_reduce_runs(const K* __restrict__ keys, const W* __restrict__ w, uint64_t n, K* __restrict__ out,
                  W* __restrict__ out_w, const uint64_t* __restrict__ rank0, uint32_t* status) {
  constexpr int RR_ITEMS = RRCfg<K, W, TROP>::ITEMS;
  constexpr uint32_t RR_TILE = RRCfg<K, W, TROP>::TILE;
  __shared__ K s_k[RR_TILE];
  __shared__ W s_w[TROP ? RR_TILE : 1];
  __shared__ K s_ok[RR_TILE];
  __shared__ W s_ow[TROP ? RR_TILE : 1];
  __shared__ uint32_t s_scan[NT / 32 + 1];
  __shared__ SegMin<W> s_seg[NT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t t0 = (uint64_t)blockIdx.x * RR_TILE;
  const uint32_t len = (uint32_t)(n - t0 < RR_TILE ? n - t0 : RR_TILE);
  const uint64_t base = rank0[blockIdx.x];  // output rank of this tile's first head
#pragma unroll
  for (int q = 0; q < RR_ITEMS; q++) {
    const uint32_t k = q * NT + tid;
    if (k < len) {
      s_k[k] = keys[t0 + k];
      if constexpr (TROP) s_w[k] = w[t0 + k];
    }
  }
  __syncthreads();
  const uint32_t b = tid * RR_ITEMS;
  bool head[RR_ITEMS], last[RR_ITEMS];
  W incl[RR_ITEMS];
  SegMin<W> run{false, W(0)};
  uint32_t nh = 0;  // heads among this thread's items
#pragma unroll
  for (int j = 0; j < RR_ITEMS; j++) {
    const uint32_t li = b + j;
    head[j] = false;
    last[j] = false;
    incl[j] = W(0);
    if (li < len) {
      const uint64_t gi = t0 + li;
      const K kk = s_k[li];
      head[j] = (gi == 0) || (kk != (li > 0 ? s_k[li - 1] : keys[gi - 1]));
      last[j] = (gi + 1 >= n) || (kk != (li + 1 < len ? s_k[li + 1] : keys[gi + 1]));
      nh += head[j] ? 1u : 0u;
      if constexpr (TROP) {
        const W wv = s_w[li];
        if (head[j]) run = SegMin<W>{true, wv};
        else if (j == 0) run = SegMin<W>{false, wv};  // partial run entering the thread
        else run = SegMin<W>{run.h, run.m < wv ? run.m : wv};
        incl[j] = run.m;
      }
    }
  }
  if constexpr (TROP) {
    // Block-wide exclusive segmented min of the thread aggregates; the tile's
    // first run part starts at the tile (nothing enters from before it).
    SegMin<W> agg = (b < len) ? run : SegMin<W>{false, WAbs<W>::v};
    SegMin<W> inc = agg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      SegMin<W> t;
      t.h = __shfl_up_sync(kFull, inc.h, o);
      t.m = __shfl_up_sync(kFull, inc.m, o);
      if (lane >= o) inc = seg_combine(t, inc);
    }
    if (lane == 31) s_seg[warp] = inc;
    __syncthreads();
    SegMin<W> wpre{false, WAbs<W>::v};
    for (int q = 0; q < warp; q++) wpre = seg_combine(wpre, s_seg[q]);
    SegMin<W> ex;
    ex.h = __shfl_up_sync(kFull, inc.h, 1);
    ex.m = __shfl_up_sync(kFull, inc.m, 1);
    if (lane == 0) ex = SegMin<W>{false, WAbs<W>::v};
    const SegMin<W> pre = seg_combine(wpre, ex);
#pragma unroll
    for (int j = 0; j < RR_ITEMS; j++) {
      if (b + j < len) {
        if (head[j]) break;
        incl[j] = pre.m < incl[j] ? pre.m : incl[j];
      }
    }
  }
  uint32_t tile_nh;
  uint32_t r = block_excl_sum<NT>(nh, s_scan, &tile_nh);  // heads in the tile before this thread
#pragma unroll
  for (int j = 0; j < RR_ITEMS; j++) {
    const uint32_t li = b + j;
    if (li >= len) continue;
    if (head[j]) {
      s_ok[r] = s_k[li];
      r++;
    }
    if constexpr (TROP) {
      // item li belongs to the tile's run r - 1, or (r == 0) to the run that
      // entered the tile from before it
      const bool tile_end = li + 1 == len;
      if (last[j] && r > 0) {
        s_ow[r - 1] = incl[j];  // a run held whole by the tile: written below
      } else if (last[j] || tile_end) {
        // the part of a run that crosses a tile boundary: merged into its slot
        const uint64_t slot = base + r - 1;  // r == 0: base >= 1 (tile 0 starts with a head)
        if (slot < n) atomic_min_w(&out_w[slot], incl[j]);
        else atomicOr(status, ST_BOUNDS);
      }
    }
  }
  __syncthreads();
  for (uint32_t k = tid; k < tile_nh; k += NT) {
    if (base + k >= n) {
      atomicOr(status, ST_BOUNDS);
      break;
    }
    out[base + k] = s_ok[k];
    if constexpr (TROP) {
      // the tile's last run is written here only if it ends inside the tile
      // (otherwise its slot is merged by atomicMin from every tile it spans)
      if (k + 1 < tile_nh || t0 + len >= n || s_k[len - 1] != keys[t0 + len]) out_w[base + k] = s_ow[k];
    }
  }
}

// ---------------------------------------------------------------------------
// merge_diff: full ∪ cand and the delta, one merge-path pass
// ---------------------------------------------------------------------------
constexpr int MD_ITEMS = 6;
constexpr uint32_t MD_TILE = NT * MD_ITEMS;

// Merge-path split of diagonal d: #A among the first d merged elements (A wins
// ties), then moved so that an equal pair A[i-1] == B[j] stays in one tile.
template <class K>
__device__ void md_split(const K* A, uint64_t na, const K* B, uint64_t nb, uint64_t d,
                         uint64_t* oi, uint64_t* oj) {
  uint64_t lo = d > nb ? d - nb : 0, hi = d < na ? d : na;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (A[mid] <= B[d - mid - 1]) lo = mid + 1; else hi = mid;
  }
  uint64_t i = lo, j = d - lo;
  if (i > 0 && j < nb && A[i - 1] == B[j]) j++;
  *oi = i;
  *oj = j;
}

// Merge-path splits of every tile boundary at once (one thread per
// diagonal): splits[2t], splits[2t+1] = md_split of diagonal min(t*MD_TILE, na+nb).
template <class K>
__global__ void k_md_bounds(const K* __restrict__ A, uint64_t na, const K* __restrict__ B, uint64_t nb,
                            uint32_t tiles, uint64_t* __restrict__ splits) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t > tiles) return;
  const uint64_t L = na + nb, d = t * MD_TILE < L ? t * MD_TILE : L;
  md_split(A, na, B, nb, d, &splits[2 * t], &splits[2 * t + 1]);
}

// Two passes over the same tiles, reduce-then-scan (no tile waits on
// another): PASS 0 counts each tile's full-out rows and Δ' rows into
// tile_full / tile_delta; after their exclusive scan, PASS 1 recomputes the tile
// and writes its rows at the scanned offsets.
template <class K, class W, bool TROP, bool WRITE_FULL, bool WRITE_DELTA, bool INPLACE, int PASS>
__global__ void __launch_bounds__(NT)
    k_merge_diff(const K* __restrict__ A, W* Aw, uint64_t na, const K* __restrict__ B,
                 const W* __restrict__ Bw, uint64_t nb, K* __restrict__ fout, W* __restrict__ fout_w,
                 K* __restrict__ dout, W* __restrict__ dout_w, const uint64_t* __restrict__ splits,
                 uint64_t* tile_full, uint64_t* tile_delta, uint32_t* status) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  constexpr uint32_t CAP = MD_TILE + 2;
  K* s_a = reinterpret_cast<K*>(s_raw);
  K* s_b = s_a + CAP;
  W* s_aw = reinterpret_cast<W*>(s_b + CAP);
  W* s_bw = s_aw + (TROP ? CAP : 0);
  uint32_t* s_mpre = reinterpret_cast<uint32_t*>(s_bw + (TROP ? CAP : 0));  // CAP + 1
  uint32_t* s_dpre = s_mpre + CAP + 1;                                      // CAP
  __shared__ uint32_t s_scan[NT / 32 + 1];
  const int tid = threadIdx.x;
  const uint32_t tile = blockIdx.x;
  const uint64_t s_r[4] = {splits[2 * tile], splits[2 * tile + 1], splits[2 * tile + 2], splits[2 * tile + 3]};
  const uint64_t i0 = s_r[0], j0 = s_r[1];
  // Impossible for sorted unique inputs; checked so unsorted input cannot
  // index past shared memory.
  const bool oversize = s_r[2] < i0 || s_r[3] < j0 || (s_r[2] - i0) > MD_TILE + 1 ||
                        (s_r[3] - j0) > MD_TILE + 1 || (s_r[2] - i0) + (s_r[3] - j0) > MD_TILE + 1;
  if (oversize && tid == 0) atomicOr(status, ST_BOUNDS);
  const uint32_t acnt = oversize ? 0u : (uint32_t)(s_r[2] - i0);
  const uint32_t bcnt = oversize ? 0u : (uint32_t)(s_r[3] - j0);
  constexpr int BI = (MD_TILE + 2 + NT - 1) / NT;
#pragma unroll
  for (int q = 0; q < BI; q++) {
    const uint32_t k = q * NT + tid;
    if (k < acnt) {
      s_a[k] = A[i0 + k];
      if constexpr (TROP) s_aw[k] = Aw[i0 + k];
    }
    if (k < bcnt) {
      s_b[k] = B[j0 + k];
      if constexpr (TROP) s_bw[k] = Bw[j0 + k];
    }
  }
  __syncthreads();
  // Per B element: rank in A, matched?, delta?
  uint32_t b_ra[BI];
  uint32_t mflag = 0, dflag = 0;  // bit per item
  uint32_t mcount = 0, dcount = 0;
  const uint32_t bb = tid * BI;
#pragma unroll
  for (int q = 0; q < BI; q++) {
    const uint32_t jb = bb + q;
    b_ra[q] = 0;
    if (jb < bcnt) {
      const K x = s_b[jb];
      uint32_t lo = 0, hi = acnt;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_a[mid] < x) lo = mid + 1; else hi = mid;
      }
      b_ra[q] = lo;
      const bool m = lo < acnt && s_a[lo] == x;
      bool dl = !m;
      if constexpr (TROP) dl = dl || (s_bw[jb] < s_aw[lo]);
      if (m) { mflag |= 1u << q; mcount++; }
      if (dl) { dflag |= 1u << q; dcount++; }
    }
  }
  uint32_t mtot, dtot;
  const uint32_t mex = block_excl_sum<NT>(mcount, s_scan, &mtot);
  const uint32_t dex = block_excl_sum<NT>(dcount, s_scan, &dtot);
  {
    uint32_t mr = mex, dr = dex;
#pragma unroll
    for (int q = 0; q < BI; q++) {
      const uint32_t jb = bb + q;
      if (jb < bcnt) {
        s_mpre[jb] = mr;
        s_dpre[jb] = dr;
        mr += (mflag >> q) & 1u;
        dr += (dflag >> q) & 1u;
      }
    }
    if (tid == 0) s_mpre[bcnt] = mtot;
  }
  const uint32_t fcnt = acnt + bcnt - mtot;
  if constexpr (PASS == 0) {
    if (tid == 0) {
      tile_full[tile] = fcnt;
      tile_delta[tile] = dtot;
    }
    return;
  }
  const uint64_t fex = tile_full[tile], dexg = tile_delta[tile];
  __syncthreads();  // every thread's s_mpre / s_dpre entries are read below
  // B elements: unmatched -> full_out; delta -> delta out.
#pragma unroll
  for (int q = 0; q < BI; q++) {
    const uint32_t jb = bb + q;
    if (jb < bcnt) {
      const bool m = (mflag >> q) & 1u;
      if (WRITE_FULL && !m) {
        const uint64_t p = fex + b_ra[q] + (jb - s_mpre[jb]);
        if (p < na + nb) {
          fout[p] = s_b[jb];
          if constexpr (TROP) fout_w[p] = s_bw[jb];
        } else {
          atomicOr(status, ST_BOUNDS);
        }
      }
      if (WRITE_DELTA && ((dflag >> q) & 1u)) {
        const uint64_t p = dexg + s_dpre[jb];
        if (p < nb) {
          dout[p] = s_b[jb];
          if constexpr (TROP) dout_w[p] = s_bw[jb];
        } else {
          atomicOr(status, ST_BOUNDS);
        }
      }
      if constexpr (TROP && INPLACE) {
        if (m && s_bw[jb] < s_aw[b_ra[q]]) Aw[i0 + b_ra[q]] = s_bw[jb];
      }
    }
  }
  if constexpr (WRITE_FULL) {
    for (uint32_t ia = tid; ia < acnt; ia += NT) {
      const K x = s_a[ia];
      uint32_t lo = 0, hi = bcnt;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_b[mid] < x) lo = mid + 1; else hi = mid;
      }
      const uint64_t p = fex + ia + (lo - s_mpre[lo]);
      if (p >= na + nb) {
        atomicOr(status, ST_BOUNDS);
        continue;
      }
      fout[p] = x;
      if constexpr (TROP) {
        W wv = s_aw[ia];
        if (lo < bcnt && s_b[lo] == x && s_bw[lo] < wv) wv = s_bw[lo];
        fout_w[p] = wv;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// plumbing kernels
// ---------------------------------------------------------------------------
template <class K>
__global__ void k_csr_offsets(const K* __restrict__ keys, uint64_t m, int vbits, uint64_t n_nodes,
                              uint32_t* __restrict__ off) {
  const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j > n_nodes) return;
  const K probe = (K)((K)j << vbits);
  uint64_t lo = 0, hi = m;
  if (j == n_nodes) { off[j] = (uint32_t)m; return; }
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (keys[mid] < probe) lo = mid + 1; else hi = mid;
  }
  off[j] = (uint32_t)lo;
}

template <class K>
__global__ void k_csr_nbr(const K* __restrict__ keys, uint64_t m, uint64_t vmask, uint32_t* __restrict__ nbr) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) nbr[i] = (uint32_t)((uint64_t)keys[i] & vmask);
}

__global__ void k_mark_ids(const uint32_t* __restrict__ a, uint64_t n, uint32_t* bitmap, uint64_t limit) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = a[i];
    if (v < limit) atomicOr(&bitmap[v >> 5], 1u << (v & 31));
  }
}

// Same marks, OR-ed first into a block-private bitmap in shared memory
// (hub ids would otherwise hammer a few global words), then flushed once.
__global__ void k_mark_ids_smem(const uint32_t* __restrict__ a, uint64_t n, uint32_t* bitmap, uint64_t limit,
                                uint64_t words) {
  extern __shared__ uint32_t s_bm[];
  for (uint64_t i = threadIdx.x; i < words; i += blockDim.x) s_bm[i] = 0;
  __syncthreads();
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = a[i];
    if (v < limit) atomicOr(&s_bm[v >> 5], 1u << (v & 31));
  }
  __syncthreads();
  for (uint64_t i = threadIdx.x; i < words; i += blockDim.x)
    if (s_bm[i]) atomicOr(&bitmap[i], s_bm[i]);
}

__global__ void k_popcount(const uint32_t* __restrict__ bitmap, uint64_t words, unsigned long long* out) {
  unsigned long long c = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (uint64_t)gridDim.x * blockDim.x)
    c += __popc(bitmap[i]);
  c = warp_sum(c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

__global__ void k_max_u32(const uint32_t* __restrict__ a, uint64_t n, uint32_t* out) {
  uint32_t m = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    m = a[i] > m ? a[i] : m;
  for (int o = 16; o > 0; o >>= 1) {
    const uint32_t t = __shfl_xor_sync(kFull, m, o);
    m = t > m ? t : m;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void k_max_abs_w(const int64_t* __restrict__ w, const uint8_t* __restrict__ inf, uint64_t n,
                            unsigned long long* out) {
  unsigned long long m = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    if (inf && inf[i]) continue;
    const int64_t v = w[i];
    const unsigned long long a = v < 0 ? (unsigned long long)0 - (unsigned long long)v : (unsigned long long)v;
    m = a > m ? a : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(kFull, m, o);
    m = t > m ? t : m;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// Signed range of the finite weights: out[0] = min, out[1] = max (as
// order-preserving unsigned images, v ^ sign bit), out[2] = 1 if any finite.
__global__ void k_w_range(const int64_t* __restrict__ w, const uint8_t* __restrict__ inf, uint64_t n,
                          unsigned long long* out) {
  unsigned long long lo = ~0ull, hi = 0ull, any = 0ull;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    if (inf && inf[i]) continue;
    const unsigned long long u = (unsigned long long)w[i] ^ 0x8000000000000000ull;
    lo = u < lo ? u : lo;
    hi = u > hi ? u : hi;
    any = 1ull;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long a = __shfl_xor_sync(kFull, lo, o), b = __shfl_xor_sync(kFull, hi, o);
    lo = a < lo ? a : lo;
    hi = b > hi ? b : hi;
    any |= __shfl_xor_sync(kFull, any, o);
  }
  if ((threadIdx.x & 31) == 0 && any) {
    atomicMin(&out[0], lo);
    atomicMax(&out[1], hi);
    atomicOr(&out[2], 1ull);
  }
}

template <class K, class W, bool TROP>
__global__ void k_pack(const uint32_t* __restrict__ c0, const uint32_t* __restrict__ c1,
                       const int64_t* __restrict__ w, const uint8_t* __restrict__ inf, uint64_t n,
                       int shift, K* __restrict__ keys, W* __restrict__ ow, int64_t wshift, uint32_t* status) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = (K)((c0 ? ((K)c0[i] << shift) : K(0)) | (K)c1[i]);  // NULL c0: unary key
  if constexpr (TROP) {
    const bool is_inf = inf && inf[i];
    const int64_t v = w ? w[i] : 0;  // NULL weights = the (x) identity Finite(0)
    if (is_inf) {
      ow[i] = WInf<W>::v;
    } else {
      // code = v - wshift; it must not wrap and must stay below the reserved codes
      const bool low = v < INT64_MIN + wshift;
      const int64_t code = low ? 0 : v - wshift;
      if (low || code > (int64_t)WFinMax<W>::v || (int64_t)(W)code != code) atomicOr(status, ST_SENTINEL);
      ow[i] = (W)code;
    }
  }
}

template <class K, class W, bool TROP>
__global__ void k_unpack(const K* __restrict__ keys, const W* __restrict__ w, uint64_t n, int shift,
                         uint32_t* __restrict__ c0, uint32_t* __restrict__ c1, int64_t* __restrict__ ow,
                         uint8_t* __restrict__ oinf, int64_t wshift) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const K k = keys[i];
  const K lowmask = shift >= (int)(8 * sizeof(K)) ? ~K(0) : (K)((K(1) << shift) - 1);
  if (c0) c0[i] = (uint32_t)((uint64_t)k >> shift);
  if (c1) c1[i] = (uint32_t)(k & lowmask);
  if constexpr (TROP) {
    const W v = w[i];
    const bool is_inf = v == WInf<W>::v;
    if (ow) ow[i] = is_inf ? 0 : (int64_t)v + wshift;
    if (oinf) oinf[i] = is_inf ? 1 : 0;
  }
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  // splitmix64 finalizer
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

template <class K, class W, bool TROP>
__global__ void k_fingerprint(const K* __restrict__ keys, const W* __restrict__ w, uint64_t n, int shift,
                              int64_t wshift, unsigned long long* out) {
  unsigned long long acc = 0;
  const K lowmask = (K)((K(1) << shift) - 1);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const K k = keys[i];
    const uint64_t src = (uint64_t)k >> shift, dst = (uint64_t)(k & lowmask);
    uint64_t h = mix64((src << 32) | dst);
    if constexpr (TROP) {
      const W v = w[i];
      // hash the finite VALUE (code + shift); +inf hashes as a fixed constant
      const uint64_t wv = v == WInf<W>::v ? 0xfffffffffffffffull : (uint64_t)((int64_t)v + wshift);
      h = mix64(h ^ mix64(wv + 0x51ull));
    }
    acc += h;
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}

// Scan of u64 values (exclusive or inclusive) through the tile-sum scan:
// per-tile partials in one pass, the tile offsets scanned, the values
// rewritten.
constexpr int SC_ITEMS = 8;
constexpr uint32_t SC_TILE = NT * SC_ITEMS;
__global__ void __launch_bounds__(NT) k_scan_part(const uint64_t* __restrict__ v, uint64_t n,
                                                  uint64_t* __restrict__ tile_sum) {
  __shared__ uint64_t s_red[NT / 32];
  const uint64_t b = (uint64_t)blockIdx.x * SC_TILE + (uint64_t)threadIdx.x * SC_ITEMS;
  uint64_t k = 0;
  for (int j = 0; j < SC_ITEMS; j++)
    if (b + j < n) k += v[b + j];
  k = warp_sum(k);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = k;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t s = 0;
    for (int w = 0; w < NT / 32; w++) s += s_red[w];
    tile_sum[blockIdx.x] = s;
  }
}
__global__ void __launch_bounds__(NT) k_scan_apply(const uint64_t* __restrict__ v, uint64_t n,
                                                   const uint64_t* __restrict__ tile_off, uint64_t* __restrict__ out,
                                                   int inclusive) {
  __shared__ uint64_t s_scan[NT / 32 + 1];
  const uint64_t b = (uint64_t)blockIdx.x * SC_TILE + (uint64_t)threadIdx.x * SC_ITEMS;
  uint64_t loc[SC_ITEMS], k = 0;
  for (int j = 0; j < SC_ITEMS; j++) {
    loc[j] = b + j < n ? v[b + j] : 0;
    k += loc[j];
  }
  uint64_t tot;
  uint64_t run = tile_off[blockIdx.x] + block_excl_sum<NT>(k, s_scan, &tot);
  for (int j = 0; j < SC_ITEMS; j++) {
    if (b + j < n) out[b + j] = inclusive ? run + loc[j] : run;
    run += loc[j];
  }
}

inline int grid_for(strata_ctx* ctx, uint64_t n, int per_block = NT) {
  uint64_t b = ceil_div(n, per_block);
  const uint64_t cap = (uint64_t)ctx->num_sms * 8;
  if (b > cap) b = cap;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

// ---------------------------------------------------------------------------
// host entry points
// ---------------------------------------------------------------------------
template <class K>
void expand_offsets(strata_ctx* ctx, const K* dkeys, uint64_t n, int jshift, uint64_t jmask,
                    const uint32_t* off, uint64_t n_nodes, uint64_t* pos, uint32_t gmax, uint64_t* cand_total) {
  if (n == 0) {
    SK_CUDA(cudaMemsetAsync(pos, 0, sizeof(uint64_t), ctx->stream));
    return;
  }
  const uint32_t tiles = (uint32_t)ceil_div(n, EO_TILE);
  DBuf<uint64_t> sums(ctx, tiles + 1);
  const int kh = kprof_begin(ctx, K_EXPAND_OFFSETS);
  // The count uses the same warp-striped item order as the write; only the
  // per-tile totals matter, so its block-strided loop is equivalent.
  k_deg_count<K><<<tiles, NT, 0, ctx->stream>>>(dkeys, n, jshift, jmask, off, n_nodes, gmax, sums.p,
                                                reinterpret_cast<unsigned long long*>(cand_total));
  k_scan_tile_sums<<<1, 1024, 0, ctx->stream>>>(sums.p, tiles);
  k_deg_write<K><<<tiles, NT, 0, ctx->stream>>>(dkeys, n, jshift, jmask, off, n_nodes, gmax, sums.p, tiles, pos);
  kprof_end(ctx, kh, 2 * n * (sizeof(K) + 8) + n * 8);
  ctx->launches += 2;
  after_launch(ctx, "k_deg_write");
}

void scan_tile_sums(strata_ctx* ctx, uint64_t* sums, uint64_t count, int arrays) {
  k_scan_tile_sums<<<arrays, 1024, 0, ctx->stream>>>(sums, count);
  after_launch(ctx, "k_scan_tile_sums");
}

template <class K, class W, bool TROP>
void expand_emit(strata_ctx* ctx, const K* dkeys, const W* dw, uint64_t n, const uint64_t* pos,
                 uint64_t total, int jshift, uint64_t jmask, int pshift, uint64_t pmask,
                 int out_pshift, int out_vshift, const uint32_t* off, uint64_t n_nodes,
                 const uint32_t* nbr, uint64_t n_nbr, const W* nbr_w, K* out, W* out_w) {
  if (total == 0 || n == 0) return;
  const uint64_t tiles = ceil_div(n + total, EE_TILE);
  if (tiles > 0x7fffffffull) fail(STRATA_E_UNSUPPORTED, "expand too large for one launch");
  const int kh = kprof_begin(ctx, K_EXPAND_EMIT);
  k_expand_emit<K, W, TROP><<<(unsigned)tiles, NT, 0, ctx->stream>>>(
      dkeys, dw, n, pos, total, jshift, jmask, pshift, pmask, out_pshift, out_vshift, off, n_nodes,
      nbr, n_nbr, nbr_w, out, out_w, ctx->wshift, ctx->d_status);
  const uint64_t wsz = TROP ? sizeof(W) : 0;
  kprof_end(ctx, kh, n * (sizeof(K) + wsz + 8 + 4) + total * (4 + wsz) + total * (sizeof(K) + wsz));
  after_launch(ctx, "k_expand_emit");
}

template <class K, class W, bool TROP>
void reduce_runs(strata_ctx* ctx, const K* keys, const W* w, uint64_t n, K* out, W* out_w,
                 uint64_t* d_count) {
  if (n == 0) {
    SK_CUDA(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), ctx->stream));
    return;
  }
  constexpr uint32_t TILE = RRCfg<K, W, TROP>::TILE;
  const uint64_t tiles = ceil_div(n, TILE);
  DBuf<uint64_t> rank0(ctx, tiles + 1);
  k_rr_heads<K, RRCfg<K, W, TROP>::ITEMS><<<(unsigned)tiles, NT, 0, ctx->stream>>>(keys, n, rank0.p);
  after_launch(ctx, "k_rr_heads");
  scan_tile_sums(ctx, rank0.p, tiles);  // exclusive; rank0[tiles] = number of runs
  if (TROP && tiles > 1) {
    k_rr_span<K, W><<<(unsigned)ceil_div(tiles, 256), 256, 0, ctx->stream>>>(keys, n, TILE, tiles, rank0.p, out_w);
    after_launch(ctx, "k_rr_span");
  }
  const int kh = kprof_begin(ctx, K_REDUCE_RUNS);
  k_reduce_runs<K, W, TROP><<<(unsigned)tiles, NT, 0, ctx->stream>>>(keys, w, n, out, out_w, rank0.p,
                                                                    ctx->d_status);
  kprof_end(ctx, kh, n * (sizeof(K) + (TROP ? sizeof(W) : 0)));  // reads; writes added on read-back
  after_launch(ctx, "k_reduce_runs");
  SK_CUDA(cudaMemcpyAsync(d_count, rank0.p + tiles, sizeof(uint64_t), cudaMemcpyDeviceToDevice, ctx->stream));
}

template <class K, class W, bool TROP, bool WF, bool WD, bool IP>
static void launch_merge(strata_ctx* ctx, const K* full, W* full_w, uint64_t nf, const K* cand,
                         const W* cand_w, uint64_t nc, K* fout, W* fout_w, K* dout, W* dout_w,
                         uint64_t* d_counts) {
  if (nf + nc == 0) {
    SK_CUDA(cudaMemsetAsync(d_counts, 0, 2 * sizeof(uint64_t), ctx->stream));
    return;
  }
  const uint32_t tiles = (uint32_t)ceil_div(nf + nc, MD_TILE);
  // per-tile counts (full, Δ'), each array tiles + 1 long for the scan total;
  // then the merge-path splits
  DBuf<uint64_t> buf(ctx, 2ull * (tiles + 1) + 2ull * (tiles + 1));
  uint64_t* fcount = buf.p;
  uint64_t* dcount = buf.p + tiles + 1;
  uint64_t* splits = buf.p + 2ull * (tiles + 1);
  k_md_bounds<K><<<(unsigned)ceil_div(tiles + 1, NT), NT, 0, ctx->stream>>>(full, nf, cand, nc, tiles, splits);
  after_launch(ctx, "k_md_bounds");
  constexpr uint32_t CAP = MD_TILE + 2;
  const size_t smem = 2 * CAP * sizeof(K) + (TROP ? 2 * CAP * sizeof(W) : 0) + (2 * CAP + 1) * sizeof(uint32_t);
  auto count = k_merge_diff<K, W, TROP, WF, WD, IP, 0>;
  auto write = k_merge_diff<K, W, TROP, WF, WD, IP, 1>;
  SK_CUDA(cudaFuncSetAttribute(count, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  SK_CUDA(cudaFuncSetAttribute(write, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int kh = kprof_begin(ctx, K_MERGE_DIFF);
  count<<<tiles, NT, smem, ctx->stream>>>(full, full_w, nf, cand, cand_w, nc, fout, fout_w, dout, dout_w, splits,
                                          fcount, dcount, ctx->d_status);
  scan_tile_sums(ctx, buf.p, tiles, 2);
  write<<<tiles, NT, smem, ctx->stream>>>(full, full_w, nf, cand, cand_w, nc, fout, fout_w, dout, dout_w, splits,
                                          fcount, dcount, ctx->d_status);
  kprof_end(ctx, kh, (nf + nc) * (sizeof(K) + (TROP ? sizeof(W) : 0)));  // reads; writes added on read-back
  after_launch(ctx, "k_merge_diff");
  ctx->launches += 1;  // the counting pass
  SK_CUDA(cudaMemcpyAsync(d_counts, fcount + tiles, sizeof(uint64_t), cudaMemcpyDeviceToDevice, ctx->stream));
  SK_CUDA(cudaMemcpyAsync(d_counts + 1, dcount + tiles, sizeof(uint64_t), cudaMemcpyDeviceToDevice, ctx->stream));
}

template <class K, class W, bool TROP>
void merge_diff(strata_ctx* ctx, const K* full, const W* full_w, uint64_t nf, const K* cand,
                const W* cand_w, uint64_t nc, K* full_out, W* full_out_w, K* delta, W* delta_w,
                uint64_t* d_counts) {
  launch_merge<K, W, TROP, true, true, false>(ctx, full, const_cast<W*>(full_w), nf, cand, cand_w, nc,
                                              full_out, full_out_w, delta, delta_w, d_counts);
}

template <class K, class W, bool TROP>
void merge_disjoint(strata_ctx* ctx, const K* a, const W* aw, uint64_t na, const K* b,
                    const W* bw, uint64_t nb, K* out, W* out_w) {
  DBuf<uint64_t> counts(ctx, 2);
  launch_merge<K, W, TROP, true, false, false>(ctx, a, const_cast<W*>(aw), na, b, bw, nb, out, out_w,
                                               nullptr, nullptr, counts.p);
}

template <class K, class W, bool TROP>
void diff_improve(strata_ctx* ctx, const K* cand, const W* cand_w, uint64_t nc, const K* full,
                  W* full_w, uint64_t nf, K* out, W* out_w, uint64_t* d_count) {
  DBuf<K> ck(ctx, nc + 1);
  DBuf<W> cw(ctx, TROP ? nc + 1 : 1);
  DBuf<uint64_t> counts(ctx, 2);
  reduce_runs<K, W, TROP>(ctx, cand, cand_w, nc, ck.p, cw.p, counts.p);
  uint64_t nu;
  read_u64(ctx, counts.p, &nu, 1);
  launch_merge<K, W, TROP, false, true, true>(ctx, full, full_w, nf, ck.p, cw.p, nu, nullptr, nullptr,
                                              out, out_w, counts.p);
  SK_CUDA(cudaMemcpyAsync(d_count, counts.p + 1, sizeof(uint64_t), cudaMemcpyDeviceToDevice, ctx->stream));
}

template <class K>
void build_csr(strata_ctx* ctx, const K* keys, uint64_t m, int vbits, uint64_t n_nodes,
               uint32_t* off, uint32_t* nbr) {
  if (m >= 0xffffffffull) fail(STRATA_E_UNSUPPORTED, "CSR limited to 2^32-1 edges");
  k_csr_offsets<K><<<(unsigned)ceil_div(n_nodes + 1, NT), NT, 0, ctx->stream>>>(keys, m, vbits, n_nodes, off);
  after_launch(ctx, "k_csr_offsets");
  if (m) {
    const uint64_t vmask = vbits >= 64 ? ~0ull : ((1ull << vbits) - 1);
    k_csr_nbr<K><<<(unsigned)ceil_div(m, NT), NT, 0, ctx->stream>>>(keys, m, vmask, nbr);
    after_launch(ctx, "k_csr_nbr");
  }
}

uint64_t count_distinct_ids(strata_ctx* ctx, const uint32_t* a, uint64_t na, const uint32_t* b,
                            uint64_t nb, const uint32_t* c, uint64_t nc, uint64_t limit) {
  if (limit == 0) return 0;
  const uint64_t words = ceil_div(limit, 32);
  DBuf<uint32_t> bm(ctx, words);
  DBuf<unsigned long long> cnt(ctx, 1);
  SK_CUDA(cudaMemsetAsync(bm.p, 0, words * 4, ctx->stream));
  SK_CUDA(cudaMemsetAsync(cnt.p, 0, 8, ctx->stream));
  const uint32_t* cols[3] = {a, b, c};
  const uint64_t ns[3] = {na, nb, nc};
  const size_t smem = words * 4;
  const bool private_bm = smem <= 160 * 1024;
  if (private_bm)
    SK_CUDA(cudaFuncSetAttribute(k_mark_ids_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (int q = 0; q < 3; q++) {
    if (!cols[q] || !ns[q]) continue;
    if (private_bm) {
      // few blocks: each flushes its whole private bitmap once
      const int blocks = (int)std::min<uint64_t>(ceil_div(ns[q], 1024 * 32), (uint64_t)ctx->num_sms);
      k_mark_ids_smem<<<blocks, 1024, smem, ctx->stream>>>(cols[q], ns[q], bm.p, limit, words);
      after_launch(ctx, "k_mark_ids_smem");
    } else {
      k_mark_ids<<<grid_for(ctx, ns[q]), NT, 0, ctx->stream>>>(cols[q], ns[q], bm.p, limit);
      after_launch(ctx, "k_mark_ids");
    }
  }
  k_popcount<<<grid_for(ctx, words), NT, 0, ctx->stream>>>(bm.p, words, cnt.p);
  after_launch(ctx, "k_popcount");
  uint64_t r;
  read_u64(ctx, reinterpret_cast<uint64_t*>(cnt.p), &r, 1);
  return r;
}

uint32_t max_u32(strata_ctx* ctx, const uint32_t* a, uint64_t n) {
  if (n == 0) return 0;
  DBuf<uint64_t> m(ctx, 1);
  SK_CUDA(cudaMemsetAsync(m.p, 0, 8, ctx->stream));
  k_max_u32<<<grid_for(ctx, n), NT, 0, ctx->stream>>>(a, n, reinterpret_cast<uint32_t*>(m.p));
  after_launch(ctx, "k_max_u32");
  uint64_t r;
  read_u64(ctx, m.p, &r, 1);
  return (uint32_t)(r & 0xffffffffull);
}

uint64_t max_abs_weight(strata_ctx* ctx, const int64_t* w, const uint8_t* inf, uint64_t n) {
  if (n == 0 || !w) return 0;
  DBuf<unsigned long long> m(ctx, 1);
  SK_CUDA(cudaMemsetAsync(m.p, 0, 8, ctx->stream));
  k_max_abs_w<<<grid_for(ctx, n), NT, 0, ctx->stream>>>(w, inf, n, m.p);
  after_launch(ctx, "k_max_abs_w");
  uint64_t r;
  read_u64(ctx, reinterpret_cast<uint64_t*>(m.p), &r, 1);
  return r;
}

bool weight_range(strata_ctx* ctx, const int64_t* w, const uint8_t* inf, uint64_t n, int64_t* mn, int64_t* mx) {
  *mn = *mx = 0;
  if (n == 0) return false;
  if (!w) return true;  // NULL weights: every fact is Finite(0)
  DBuf<unsigned long long> r(ctx, 3);
  const unsigned long long init[3] = {~0ull, 0ull, 0ull};
  SK_CUDA(cudaMemcpyAsync(r.p, init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream));
  k_w_range<<<grid_for(ctx, n), NT, 0, ctx->stream>>>(w, inf, n, r.p);
  after_launch(ctx, "k_w_range");
  uint64_t h[3];
  read_u64(ctx, reinterpret_cast<uint64_t*>(r.p), h, 3);
  if (!h[2]) return false;
  *mn = (int64_t)(h[0] ^ 0x8000000000000000ull);
  *mx = (int64_t)(h[1] ^ 0x8000000000000000ull);
  return true;
}

template <class K, class W, bool TROP>
void pack_pairs(strata_ctx* ctx, const uint32_t* c0, const uint32_t* c1, const int64_t* w,
                const uint8_t* inf, uint64_t n, int shift, K* keys, W* ow) {
  if (n == 0) return;
  k_pack<K, W, TROP><<<(unsigned)ceil_div(n, NT), NT, 0, ctx->stream>>>(c0, c1, w, inf, n, shift, keys, ow,
                                                                       ctx->wshift, ctx->d_status);
  after_launch(ctx, "k_pack");
}

template <class K, class W, bool TROP>
void unpack_pairs(strata_ctx* ctx, const K* keys, const W* w, uint64_t n, int shift, uint32_t* c0,
                  uint32_t* c1, int64_t* ow, uint8_t* oinf) {
  if (n == 0) return;
  k_unpack<K, W, TROP><<<(unsigned)ceil_div(n, NT), NT, 0, ctx->stream>>>(keys, w, n, shift, c0, c1, ow, oinf,
                                                                         ctx->wshift);
  after_launch(ctx, "k_unpack");
}

template <class K, class W, bool TROP>
uint64_t fingerprint(strata_ctx* ctx, const K* keys, const W* w, uint64_t n, int shift) {
  DBuf<unsigned long long> acc(ctx, 1);
  SK_CUDA(cudaMemsetAsync(acc.p, 0, 8, ctx->stream));
  if (n) {
    k_fingerprint<K, W, TROP><<<grid_for(ctx, n), NT, 0, ctx->stream>>>(keys, w, n, shift, ctx->wshift, acc.p);
    after_launch(ctx, "k_fingerprint");
  }
  uint64_t r;
  read_u64(ctx, reinterpret_cast<uint64_t*>(acc.p), &r, 1);
  return r;
}

void scan_u64(strata_ctx* ctx, const uint64_t* v, uint64_t n, uint64_t* out, bool inclusive, uint64_t* total) {
  const uint64_t tiles = ceil_div(n ? n : 1, SC_TILE);
  DBuf<uint64_t> ts(ctx, tiles + 1);
  k_scan_part<<<(unsigned)tiles, NT, 0, ctx->stream>>>(v, n, ts.p);
  after_launch(ctx, "k_scan_part");
  scan_tile_sums(ctx, ts.p, tiles);
  k_scan_apply<<<(unsigned)tiles, NT, 0, ctx->stream>>>(v, n, ts.p, out, inclusive ? 1 : 0);
  after_launch(ctx, "k_scan_apply");
  if (total) read_u64(ctx, ts.p + tiles, total, 1);
}

// ---- explicit instantiations ----------------------------------------------------
template void expand_offsets<uint32_t>(strata_ctx*, const uint32_t*, uint64_t, int, uint64_t, const uint32_t*, uint64_t,
                                       uint64_t*, uint32_t, uint64_t*);
template void expand_offsets<uint64_t>(strata_ctx*, const uint64_t*, uint64_t, int, uint64_t, const uint32_t*, uint64_t,
                                       uint64_t*, uint32_t, uint64_t*);
template void build_csr<uint32_t>(strata_ctx*, const uint32_t*, uint64_t, int, uint64_t, uint32_t*, uint32_t*);
template void build_csr<uint64_t>(strata_ctx*, const uint64_t*, uint64_t, int, uint64_t, uint32_t*, uint32_t*);

#define SK_INST_KW(K, W, T)                                                                          \
  template void expand_emit<K, W, T>(strata_ctx*, const K*, const W*, uint64_t, const uint64_t*,     \
                                     uint64_t, int, uint64_t, int, uint64_t, int, int,               \
                                     const uint32_t*, uint64_t, const uint32_t*, uint64_t, const W*, \
                                     K*, W*);                                                        \
  template void reduce_runs<K, W, T>(strata_ctx*, const K*, const W*, uint64_t, K*, W*, uint64_t*);  \
  template void merge_diff<K, W, T>(strata_ctx*, const K*, const W*, uint64_t, const K*, const W*,   \
                                    uint64_t, K*, W*, K*, W*, uint64_t*);                            \
  template void merge_disjoint<K, W, T>(strata_ctx*, const K*, const W*, uint64_t, const K*,         \
                                        const W*, uint64_t, K*, W*);                                 \
  template void diff_improve<K, W, T>(strata_ctx*, const K*, const W*, uint64_t, const K*, W*,       \
                                      uint64_t, K*, W*, uint64_t*);                                  \
  template void pack_pairs<K, W, T>(strata_ctx*, const uint32_t*, const uint32_t*, const int64_t*,   \
                                    const uint8_t*, uint64_t, int, K*, W*);                          \
  template void unpack_pairs<K, W, T>(strata_ctx*, const K*, const W*, uint64_t, int, uint32_t*,     \
                                      uint32_t*, int64_t*, uint8_t*);                                \
  template uint64_t fingerprint<K, W, T>(strata_ctx*, const K*, const W*, uint64_t, int);
SK_INST_KW(uint32_t, int32_t, false)
SK_INST_KW(uint64_t, int32_t, false)
SK_INST_KW(uint32_t, int32_t, true)
SK_INST_KW(uint64_t, int32_t, true)
SK_INST_KW(uint32_t, int64_t, true)
SK_INST_KW(uint64_t, int64_t, true)
#undef SK_INST_KW

}  // namespace sk
