// sk_dense.cu — the direct-addressed plan of the semi-naive round.
//
// When the product of the two column domains is small enough (the
// benchmark's dist(S, Z): 64 × 552,101), a relation is held as a dense
// index over (c0, c1): a membership bitmap for Bool, an int32 weight array
// for Trop (ABSENT = INT32_MAX, +inf = INT32_MAX-1).  One round then needs no
// sort and no merge:
//
//   for every candidate (entry, w) of Δ ⋈ E:            (load-balanced expand)
//     Bool:  if entry absent from the value read:  set bit, set mark
//     Trop:  if w < the value read:  atomicMin(D[entry], w), set mark
//   Δ' = the marked entries; their merged weights are D at the round's end
//
// An entry is marked exactly when it is new (Bool) or strictly below the
// value it had when the round started (Trop): the interpreter's
// `Relation::combine` change test (strata-eval/src/store.rs:34-48), and Δ'
// carries the merged values (seminaive.rs:199-206), so rounds, Δ sets and
// the round cap equal the sort-merge plan's.
//
// Layout.  The index is stored as rows of the column the NEXT round joins on
// (c0 for TC's Δ(Y,Z), c1 for MSSP's Δ(S,Y)), each row padded to a multiple
// of 32 entries, so a 32-bit word of the marks holds Δ tuples of one join
// value.  Δ stays in the marks: each round compacts the nonzero marks words
// of rows with edges into word heads (dense_word_heads; the heads' weights
// are copied to Dprev, which the expand reads while D changes), and the
// expand reads each edge of a join value once for all members of a head,
// whose probes of that edge fall in one index row (cache-resident).  Only
// the bootstrap round expands a Δ given as keys (dense_heads).
#include <type_traits>

#include "sk_ops.cuh"
#include "sk_prims.cuh"

namespace sk {
namespace {

constexpr int NT = 256;
constexpr int DE_ITEMS = 8;
constexpr uint32_t DE_TILE = NT * DE_ITEMS;
constexpr uint32_t kGroupMax = 32;  // group members per expand output (runs are split at multiples of 32)

__device__ __forceinline__ uint64_t mp_before(const uint64_t* pos, uint64_t n, uint64_t d) {
  uint64_t lo = 0, hi = d < n ? d : n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (mid + pos[mid] < d) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// splits[t] = #Δ items whose event precedes merged index t*tile (t <= tiles).
__global__ void k_tile_splits(const uint64_t* __restrict__ pos, uint64_t n, uint64_t total, uint32_t tile,
                              uint64_t tiles, uint64_t* __restrict__ splits) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t > tiles) return;
  const uint64_t L = n + total;
  uint64_t d = t * (uint64_t)tile;
  if (d > L) d = L;
  splits[t] = mp_before(pos, n, d);
}

__device__ __forceinline__ uint64_t dense_index(uint64_t key, const DenseLayout& L) {
  const uint64_t c0 = key >> L.b1, c1 = key & L.mask1;
  return L.colmajor ? c1 * L.width + c0 : c0 * L.width + c1;
}

// Position of the k-th (0-based) set bit of w (k < popc(w)).
__device__ __forceinline__ uint32_t select_bit(uint32_t w, uint32_t k) {
  uint32_t pos = 0;
#pragma unroll
  for (int sh = 16; sh >= 1; sh >>= 1) {
    const uint32_t c = __popc((w >> pos) & ((1u << sh) - 1u));
    if (k >= c) {
      k -= c;
      pos += sh;
    }
  }
  return pos;
}

// Grouped expand over compacted group heads.  A head is either
//   * a key head (dense_heads): a run of Δ rows with one join value, split
//     at multiples of kGroupMax; its members are the rows h .. h+g-1, or
//   * a word head (dense_word_heads): a nonzero 32-bit word of the marks in
//     the index row of one join value; its members are the word's set bits,
//     their weights in Dprev,
// and carries the degree of its join value, so one expand output is one
// (head, edge) pair and the load balancing spends no merged positions on the
// other members.  A warp takes 32 consecutive outputs (one per lane) and
// flattens their (edge, member) candidates: each lane writes one slot per
// member of its output into the warp's slot table, (lane << 5) | member, at
// its exclusive prefix of the group sizes, and the warp then processes the
// slots 32 at a time.  Lanes that share an edge handle consecutive members
// of its group, whose index entries are adjacent in one index row, so a
// warp's probes and atomics touch one or two cache lines instead of 32.
//
// Marks.  A candidate marks its entry when it is below (Trop) or absent
// from (Bool) the value the candidate read, and then merges with an atomic
// whose result it does not wait for.  An entry is marked exactly when it
// changed this round: a value read during the round is at most the round's
// starting value, and the first candidate that lowers (sets) an entry read
// the starting value, since only such candidates change it.
//
// Every head has at least one edge, so the head events of a tile's 2,048
// merged positions are at least two apart: a tile sees at most
// DE_TILE / 2 + 1 heads (checked).
constexpr uint32_t DE_HEADS = DE_TILE / 2 + 2;
constexpr uint32_t kWarps = NT / 32;
// Word heads with at least this many members take the bit-lane path (one
// warp iteration per output at popc / 32 lane use, no slot lookups); the
// sparser ones are flattened.  Tunable (STRATA_KNOB_DENSE_WORD_MEMBERS).
constexpr int kDenseMembers = 24;

// 64-bit atomic minimum for the wide lanes.
__device__ __forceinline__ void atomic_min_w(int32_t* p, int32_t v) { atomicMin(p, v); }
__device__ __forceinline__ void atomic_min_w(int64_t* p, int64_t v) {
  atomicMin(reinterpret_cast<long long*>(p), (long long)v);
}

template <class K, bool TROP, bool WORDS, class IX, class W>
__global__ void __launch_bounds__(NT, 5)
    k_expand_dense(const K* __restrict__ dkeys, const W* __restrict__ dw, uint64_t n_rows,
                   const uint32_t* __restrict__ hidx, const uint64_t* __restrict__ pos,
                   const uint32_t* __restrict__ hseg, const typename std::conditional<WORDS, uint32_t, uint8_t>::type* __restrict__ hg,
                   uint64_t n, uint64_t total, const uint64_t* __restrict__ splits, int pshift, uint64_t pmask,
                   uint64_t ck, uint64_t cv, uint32_t wpr, int wpr_shift, int dense_members,
                   const uint32_t* __restrict__ nbr,
                   uint64_t n_nbr,
                   const W* __restrict__ nbr_w, uint64_t entries, uint32_t* bits, W* D, uint32_t* marks,
                   int64_t wshift, uint32_t* status) {
  using GT = typename std::conditional<WORDS, uint32_t, uint8_t>::type;
  // IX: the index type of entries (32-bit when the index has < 2^32 entries)
  const IX ckx = (IX)ck;
  // Dynamic shared memory (sizes in dense_expand_smem()):
  //   s_pos   int32  pos of each local head relative to the tile's first output
  //   s_seg   u32    CSR segment start of each local head
  //   s_h     u32    Δ row (key head) or marks word (word head) of each local head
  //   s_g     u8/u32 group size (key head) or member mask (word head)
  //   s_owner u16    local owner head of each output of the tile
  //   s_slot  u16    per warp: the (lane, member) of each candidate of its chunk
  extern __shared__ __align__(16) unsigned char s_raw[];
  int32_t* s_pos = reinterpret_cast<int32_t*>(s_raw);
  uint32_t* s_seg = reinterpret_cast<uint32_t*>(s_pos + DE_HEADS);
  uint32_t* s_h = s_seg + DE_HEADS;
  GT* s_g = reinterpret_cast<GT*>(s_h + DE_HEADS);
  uint16_t* s_owner = reinterpret_cast<uint16_t*>(s_g + DE_HEADS);
  uint16_t* s_slot = s_owner + DE_TILE;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint16_t* my_slots = s_slot + warp * (32 * kGroupMax);
  const uint64_t L = n + total;
  const uint64_t d0 = (uint64_t)blockIdx.x * DE_TILE;
  const uint64_t d1 = d0 + DE_TILE < L ? d0 + DE_TILE : L;
  const uint64_t i0 = splits[blockIdx.x], i1 = splits[blockIdx.x + 1];
  const uint64_t a = i0 > 0 ? i0 - 1 : 0;
  if (i1 < a || i1 - a > DE_HEADS || i1 > n || d1 < i1 || d0 < i0) {
    if (tid == 0) atomicOr(status, ST_BOUNDS);
    return;
  }
  const uint64_t o0 = d0 - i0, o1 = d1 - i1;
  const uint32_t cnt = (uint32_t)(i1 - a);
  for (uint32_t k = tid; k < cnt; k += NT) {
    const uint64_t i = a + k;
    const int64_t rel = (int64_t)pos[i] - (int64_t)o0;  // one head's degree stays below 2^31
    if (rel < INT32_MIN || rel > INT32_MAX) atomicOr(status, ST_BOUNDS);
    s_pos[k] = (int32_t)rel;
    s_seg[k] = hseg[i];
    s_h[k] = hidx[i];
    s_g[k] = hg[i];
  }
  __syncthreads();
  uint32_t flags = 0;
  // Serial merge of item events and outputs: thread t walks merged positions
  // [d0 + t*ITEMS, ...) once and records the owner of every output it meets.
  // Item a+k sits at merged position (a+k) + pos[a+k]; output o owned by
  // item i sits at o + i + 1.
  {
    const uint64_t p0 = d0 + (uint64_t)tid * DE_ITEMS;
    if (p0 < d1) {
      uint32_t lo = 0, hi = cnt;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((int64_t)(a + mid + o0) + s_pos[mid] < (int64_t)p0) lo = mid + 1; else hi = mid;
      }
      uint32_t kk = lo;  // local items whose event precedes p0
      const uint64_t p1 = p0 + DE_ITEMS < d1 ? p0 + DE_ITEMS : d1;
      for (uint64_t p = p0; p < p1; p++) {
        if (kk < cnt && (int64_t)(a + kk + o0) + s_pos[kk] == (int64_t)p) {
          kk++;
        } else {
          const uint64_t o = p - (a + kk);
          if (kk == 0 || o < o0 || o - o0 >= DE_TILE) flags |= ST_BOUNDS;
          else s_owner[o - o0] = (uint16_t)(kk - 1);
        }
      }
    }
  }
  __syncthreads();
  const uint64_t o_end = o1 < total ? o1 : total;
  for (uint64_t c = o0 + (uint64_t)warp * 32; c < o_end; c += NT) {
    const uint64_t o = c + lane;
    uint32_t mm = 0, v = 0;
    W ew = 0;
    uint64_t h = 0, kb = 0;
    if (o < o_end) {
      const uint32_t li = s_owner[o - o0];
      const uint64_t e = (uint64_t)((int64_t)s_seg[li] + ((int64_t)(o - o0) - s_pos[li]));
      if (li >= cnt || e >= n_nbr) {
        flags |= ST_BOUNDS;
      } else {
        v = nbr[e];
        if constexpr (TROP) ew = nbr_w[e];
        h = s_h[li];
        if constexpr (WORDS) {
          // members: the set bits of word h, columns (h mod wpr)*32 + bit of
          // the head's row; kb = the output index of column 0 of the word
          mm = s_g[li];
          const uint32_t wcol = wpr_shift >= 0 ? ((uint32_t)h & (wpr - 1u)) : (uint32_t)h % wpr;
          kb = (uint64_t)(wcol * 32u) * ck + (uint64_t)v * cv;
          // every member's entry (and Dprev slot) inside the index: checked
          // once here for the highest member
          if (h * 32 + 32 > entries || (mm && kb + (uint64_t)(31 - __clz(mm)) * ck >= entries)) {
            flags |= ST_BOUNDS;
            mm = 0;
          }
        } else {
          const uint32_t g = s_g[li];
          mm = g >= 32 ? kFull : (1u << g) - 1u;  // members h + r for the set bits r
          if (g > kGroupMax || h + g > n_rows) {
            flags |= ST_BOUNDS;
            mm = 0;
          }
        }
      }
    }
    if constexpr (WORDS) {
      // Dense words: lane l takes member bit l, and the warp walks the
      // outputs (edges) of the dense lanes several at a time; each output's
      // member weights and probes are one coalesced line.
      const uint32_t md = mm;
      unsigned dm = __ballot_sync(kFull, __popc(md) >= dense_members);
      if ((dm >> lane) & 1u) mm = 0;  // the flattened pass below takes the rest
      while (dm) {
        // outputs in flight: four with 32-bit indices and weights, two
        // otherwise (more would spill under the 51-register bound of five
        // blocks per SM)
        constexpr int U = (sizeof(IX) == 4 && sizeof(W) == 4) ? 4 : 2;
        int t[U];
        bool live[U];
        t[0] = __ffs(dm) - 1;
        live[0] = true;
        dm &= dm - 1;
#pragma unroll
        for (int u = 1; u < U; u++) {
          live[u] = dm != 0;
          t[u] = live[u] ? __ffs(dm) - 1 : t[0];
          dm &= dm - 1;
        }
        bool act[U];
        IX ixd[U];
        W cwd[U], curd[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const uint32_t m_t = __shfl_sync(kFull, md, t[u]);
          const IX kb_t = __shfl_sync(kFull, (IX)kb, t[u]);
          const W ew_t = TROP ? __shfl_sync(kFull, ew, t[u]) : W(0);
          const uint32_t w_t = TROP ? __shfl_sync(kFull, (uint32_t)h, t[u]) : 0u;
          act[u] = ((m_t >> lane) & 1u) && live[u];
          ixd[u] = kb_t + (IX)lane * ckx;
          cwd[u] = 0;
          if constexpr (TROP)
            if (act[u]) cwd[u] = dw[(IX)w_t * 32 + (IX)lane];
          if (act[u]) {
            if constexpr (TROP) curd[u] = D[ixd[u]];
            else curd[u] = (W)bits[ixd[u] >> 5];
          }
          if constexpr (TROP) cwd[u] = trop_mul(cwd[u], ew_t, wshift, &flags);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
          if (!act[u]) continue;
          const uint32_t bit = 1u << (ixd[u] & 31);
          if constexpr (TROP) {
            if (cwd[u] < curd[u]) {
              atomic_min_w(&D[ixd[u]], cwd[u]);
              atomicOr(&marks[ixd[u] >> 5], bit);
            }
          } else {
            if (((uint32_t)curd[u] & bit) == 0) {
              atomicOr(&bits[ixd[u] >> 5], bit);
              atomicOr(&marks[ixd[u] >> 5], bit);
            }
          }
        }
      }
    }
    const uint32_t g = __popc(mm);
    const uint32_t incl = warp_incl_sum(g);
    const uint32_t T = __shfl_sync(kFull, incl, 31);
    {
      uint32_t k = incl - g;
      for (uint32_t r = mm; r; r &= r - 1) my_slots[k++] = (uint16_t)((lane << 5) | (__ffs(r) - 1));
    }
    __syncwarp();
    // Candidates j = 0..T-1 of this chunk: slot j names the owner lane t and
    // the member (row offset or bit) of t's head; the edge is v_t.  Four
    // candidates per lane in flight: their index probes overlap (measured
    // 3 % faster on MSSP R-MAT-20 than two, together with five resident
    // blocks of up to 51 registers instead of six of 40).
    for (uint32_t b0 = 0; b0 < T; b0 += 128) {
      IX ix[4];
      W cw[4], cur[4];
      bool ok[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const uint32_t j = b0 + 32 * u + lane;
        ok[u] = j < T;
        const uint32_t sl = ok[u] ? my_slots[j] : 0u;
        const int t = (int)(sl >> 5);
        const uint32_t r = sl & 31u;
        const W ew_t = TROP ? __shfl_sync(kFull, ew, t) : W(0);
        ix[u] = 0;
        cw[u] = 0;
        if constexpr (WORDS) {
          const IX kb_t = __shfl_sync(kFull, (IX)kb, t);
          const uint32_t w_t = TROP ? __shfl_sync(kFull, (uint32_t)h, t) : 0u;
          if (ok[u]) {
            ix[u] = kb_t + (IX)r * ckx;  // inside the index: checked per output
            if constexpr (TROP) cw[u] = trop_mul(dw[(IX)w_t * 32 + (IX)r], ew_t, wshift, &flags);
          }
        } else {
          const uint64_t h_t = __shfl_sync(kFull, h, t);
          const uint32_t v_t = __shfl_sync(kFull, v, t);
          if (ok[u]) {
            const uint64_t m = h_t + r;
            const K mk = dkeys[m];
            const uint32_t kept = (uint32_t)((mk >> pshift) & (K)pmask);
            // index of the output key (kept, v) without packing it: one of
            // the two coefficients is 1, the other the index's row width
            const uint64_t ix64 = (uint64_t)kept * ck + (uint64_t)v_t * cv;
            ix[u] = (IX)ix64;
            if (ix64 >= entries) {
              flags |= ST_BOUNDS;
              ok[u] = false;
            } else if constexpr (TROP) {
              cw[u] = trop_mul(dw[m], ew_t, wshift, &flags);
            }
          }
        }
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        if (ok[u]) {
          if constexpr (TROP) cur[u] = D[ix[u]];
          else cur[u] = (W)bits[ix[u] >> 5];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        if (!ok[u]) continue;
        const uint32_t bit = 1u << (ix[u] & 31);
        if constexpr (TROP) {
          if (cw[u] < cur[u]) {
            atomic_min_w(&D[ix[u]], cw[u]);
            atomicOr(&marks[ix[u] >> 5], bit);  // changed this round
          }
        } else {
          if (((uint32_t)cur[u] & bit) == 0) {
            atomicOr(&bits[ix[u] >> 5], bit);
            atomicOr(&marks[ix[u] >> 5], bit);  // new this round
          }
        }
      }
    }
    __syncwarp();  // the slot table is rewritten for the next chunk
  }
  if (flags) atomicOr(status, flags);
}

// The set bits of a bitmap over an index, as keys in index order (with their
// weight from D for Trop); the bitmap is cleared.  The bit-row plan turns its
// final path rows into the sorted relation with it.  Reduce-then-scan:
// per-tile counts, one-block scan, then the write (no waiting between tiles).
constexpr uint32_t MC_TILE = NT;  // bitmap words per tile (one per thread)

__global__ void __launch_bounds__(NT) k_marks_count(const uint32_t* __restrict__ marks, uint64_t words,
                                                    uint64_t* __restrict__ tile_sums) {
  __shared__ uint32_t s_red[NT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t w = (uint64_t)blockIdx.x * MC_TILE + tid;
  uint32_t c = (w < words) ? __popc(marks[w]) : 0u;
  c = warp_sum(c);
  if (lane == 0) s_red[warp] = c;
  __syncthreads();
  if (tid == 0) {
    uint64_t t = 0;
    for (int q = 0; q < NT / 32; q++) t += s_red[q];
    tile_sums[blockIdx.x] = t;
  }
}

// Each warp enumerates the set bits of its 32 words in index order, 32 at a
// time across the lanes, so the key stores and the weight gathers coalesce.
template <class K, bool TROP, class W>
__global__ void __launch_bounds__(NT)
    k_marks_write(uint32_t* marks, uint64_t words, DenseLayout lay, const W* __restrict__ D,
                  K* __restrict__ out, W* __restrict__ out_w, uint64_t out_cap,
                  const uint64_t* __restrict__ tile_sums, uint32_t* status) {
  __shared__ uint32_t s_scan[NT / 32 + 1];
  const int tid = threadIdx.x, lane = tid & 31;
  const uint64_t wi = (uint64_t)blockIdx.x * MC_TILE + tid;
  const uint32_t m = (wi < words) ? marks[wi] : 0u;
  const uint32_t c = __popc(m);
  uint32_t tot;
  const uint32_t ex = block_excl_sum<NT>(c, s_scan, &tot);
  const uint32_t incl = warp_incl_sum(c);
  const uint32_t wtot = __shfl_sync(kFull, incl, 31);
  const uint64_t wbase = tile_sums[blockIdx.x] + __shfl_sync(kFull, ex, 0);
  const uint64_t width = lay.width;
  const uint64_t b = wi * 32;
  const uint64_t row_b = b / width, col_b = b - row_b * width;  // one division per word
  uint32_t flags = 0;
  for (uint32_t s0 = 0; s0 < wtot; s0 += 32) {
    const uint32_t slot = s0 + lane;
    // owner lane = number of lanes whose inclusive count is <= slot
    int t = 0;
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) {
      const uint32_t v = __shfl_sync(kFull, incl, t + sh - 1);
      if (v <= slot) t += sh;
    }
    t &= 31;
    const uint32_t ex_t = __shfl_sync(kFull, incl - c, t);
    const uint32_t mw = __shfl_sync(kFull, m, t);
    const uint64_t rb = __shfl_sync(kFull, row_b, t), cb = __shfl_sync(kFull, col_b, t);
    const uint64_t wt = __shfl_sync(kFull, wi, t);
    if (slot < wtot) {
      const uint32_t bit = select_bit(mw, slot - ex_t);
      uint64_t row = rb, col = cb + bit;
      while (col >= width) {
        col -= width;
        row++;
      }
      const uint64_t ix = wt * 32 + bit;
      const uint64_t at = wbase + slot;
      if (ix >= lay.entries || at >= out_cap) {
        flags |= ST_BOUNDS;
      } else {
        const uint64_t c0 = lay.colmajor ? col : row, c1 = lay.colmajor ? row : col;
        out[at] = (K)(((K)c0 << lay.b1) | (K)c1);
        if constexpr (TROP) out_w[at] = D[ix];
      }
    }
  }
  if (m) marks[wi] = 0u;
  if (flags) atomicOr(status, flags);
}

// Seed the index from keys (and weights).
template <class K, bool TROP, class W>
__global__ void k_dense_seed(const K* __restrict__ keys, const W* __restrict__ w, uint64_t n,
                             DenseLayout lay, uint32_t* bits, W* D, uint32_t* marks, uint32_t* status) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t c0 = (uint64_t)keys[i] >> lay.b1, c1 = (uint64_t)keys[i] & lay.mask1;
  if (c0 >= lay.n0 || c1 >= lay.n1) { atomicOr(status, ST_BOUNDS); return; }
  const uint64_t ix = dense_index((uint64_t)keys[i], lay);
  if constexpr (TROP) D[ix] = w[i];
  else atomicOr(&bits[ix >> 5], 1u << (ix & 31));
  if (marks) atomicOr(&marks[ix >> 5], 1u << (ix & 31));
}

template <class W>
__global__ void k_fill_w(W* p, uint64_t n, W v) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

// The final relation of a row-major index, in key order (= index order):
// ordinal q enumerates (c0, c1) row-major.
constexpr int DC_ITEMS = 8;
constexpr uint32_t DC_TILE = NT * DC_ITEMS;

template <class K, bool TROP, class W>
__global__ void __launch_bounds__(NT)
    k_dense_compact(const uint32_t* __restrict__ bits, const W* __restrict__ D, DenseLayout lay,
                    K* __restrict__ out, W* __restrict__ out_w, uint64_t out_cap, uint64_t* states,
                    uint32_t* counter, uint64_t* d_count, uint32_t* status) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_scan[NT / 32 + 1];
  __shared__ uint64_t s_ex;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t tile = claim_tile(counter, &s_tile);
  const uint64_t b = (uint64_t)tile * DC_TILE + (uint64_t)tid * DC_ITEMS;
  uint32_t present = 0;
  W wv[DC_ITEMS];
  // (c0, c1) of ordinal b, then stepped: one division per thread.
  const uint64_t logical = lay.n0 * lay.n1;
  uint64_t q0 = b / lay.n1, q1 = b - q0 * lay.n1;
#pragma unroll
  for (int j = 0; j < DC_ITEMS; j++) {
    const uint64_t q = b + j;
    bool p = false;
    wv[j] = 0;
    if (j) {
      if (++q1 == lay.n1) {
        q1 = 0;
        q0++;
      }
    }
    if (q < logical) {
      const uint64_t ix = lay.colmajor ? q1 * lay.width + q0 : q0 * lay.width + q1;
      if constexpr (TROP) {
        wv[j] = D[ix];
        p = wv[j] != WAbs<W>::v;
      } else {
        p = (bits[ix >> 5] >> (ix & 31)) & 1u;
      }
    }
    present |= (p ? 1u : 0u) << j;
  }
  uint32_t tot;
  const uint32_t ex = block_excl_sum<NT>((uint32_t)__popc(present), s_scan, &tot);
  if (warp == 0) {
    const uint64_t e = warp_lookback(states, tile, tot, status);
    if (lane == 0) {
      s_ex = e;
      if (tile == gridDim.x - 1) *d_count = e + tot;
    }
  }
  __syncthreads();
  uint64_t at = s_ex + ex;
  uint64_t c0 = b / lay.n1, c1 = b - c0 * lay.n1;
#pragma unroll
  for (int j = 0; j < DC_ITEMS; j++) {
    if (j) {
      if (++c1 == lay.n1) {
        c1 = 0;
        c0++;
      }
    }
    if ((present >> j) & 1u) {
      if (at < out_cap) {
        out[at] = (K)(((K)c0 << lay.b1) | (K)c1);
        if constexpr (TROP) out_w[at] = wv[j];
      } else {
        atomicOr(status, ST_BOUNDS);
      }
      at++;
    }
  }
}

// ---- final relation of a column-major index ---------------------------------
// Key order (c0 major) runs down the columns of a column-major index, so
// enumerating it in key order strides one row width per entry.  Instead a
// warp reads a 32-row × 32-column sub-tile along its rows (lane = column,
// coalesced): the first pass records, per (column, tile of 32 rows), the
// rows present as a mask; the masks' popcounts are scanned in key order
// (column major); the second pass re-reads the sub-tile, transposes it
// through shared memory and writes each column's present entries as one
// contiguous run of keys (and weights).
constexpr int CM_ITEMS = 8;
constexpr uint32_t CM_CHUNK = NT * CM_ITEMS;  // masks per scan block

template <bool TROP, class W>
__device__ __forceinline__ bool cm_present(const uint32_t* bits, const W* D, uint64_t ix) {
  if constexpr (TROP) return D[ix] != WAbs<W>::v;
  else return (bits[ix >> 5] >> (ix & 31)) & 1u;
}

template <bool TROP, class W>
__global__ void __launch_bounds__(NT)
    k_cm_masks(const uint32_t* __restrict__ bits, const W* __restrict__ D, DenseLayout lay, uint64_t T,
               uint64_t subtiles, uint32_t* __restrict__ masks) {
  const uint64_t g = ((uint64_t)blockIdx.x * NT + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (g >= subtiles) return;
  const uint64_t cw = lay.width / 32, t = g / cw, c = (g - t * cw) * 32 + lane;
  uint32_t m = 0;
#pragma unroll 8
  for (int r = 0; r < 32; r++) {
    const uint64_t row = t * 32 + r;
    if (row < lay.rows && cm_present<TROP, W>(bits, D, row * lay.width + c)) m |= 1u << r;
  }
  if (c < lay.n0) masks[c * T + t] = m;
}

__global__ void __launch_bounds__(NT) k_cm_chunk_sums(const uint32_t* __restrict__ masks, uint64_t M,
                                                      uint64_t* __restrict__ sums) {
  __shared__ uint32_t s_red[NT / 32];
  const uint64_t b = (uint64_t)blockIdx.x * CM_CHUNK + (uint64_t)threadIdx.x * CM_ITEMS;
  uint32_t c = 0;
#pragma unroll
  for (int j = 0; j < CM_ITEMS; j++)
    if (b + j < M) c += __popc(masks[b + j]);
  c = warp_sum(c);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t t = 0;
    for (int w = 0; w < NT / 32; w++) t += s_red[w];
    sums[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(NT) k_cm_offsets(const uint32_t* __restrict__ masks, uint64_t M,
                                                   const uint64_t* __restrict__ sums, uint64_t* __restrict__ offs) {
  __shared__ uint32_t s_scan[NT / 32 + 1];
  const uint64_t b = (uint64_t)blockIdx.x * CM_CHUNK + (uint64_t)threadIdx.x * CM_ITEMS;
  uint32_t pc[CM_ITEMS], c = 0;
#pragma unroll
  for (int j = 0; j < CM_ITEMS; j++) {
    pc[j] = b + j < M ? __popc(masks[b + j]) : 0u;
    c += pc[j];
  }
  uint32_t tot;
  uint64_t run = sums[blockIdx.x] + block_excl_sum<NT>(c, s_scan, &tot);
#pragma unroll
  for (int j = 0; j < CM_ITEMS; j++) {
    if (b + j < M) offs[b + j] = run;
    run += pc[j];
  }
}

// Shared memory of k_cm_write: one 32 x 33 weight tile per warp (dynamic, so
// the 64-bit lanes' 67.6 KB fit).
template <class W>
constexpr size_t cm_write_smem() { return (size_t)(NT / 32) * 32 * 33 * sizeof(W); }

template <class K, bool TROP, class W>
__global__ void __launch_bounds__(NT)
    k_cm_write(const uint32_t* __restrict__ bits, const W* __restrict__ D, DenseLayout lay, uint64_t T,
               uint64_t subtiles, const uint32_t* __restrict__ masks, const uint64_t* __restrict__ offs,
               K* __restrict__ out, W* __restrict__ out_w, uint64_t out_cap, uint32_t* status) {
  extern __shared__ __align__(16) unsigned char s_cm_raw[];
  W (*s_w)[32][33] = reinterpret_cast<W (*)[32][33]>(s_cm_raw);
  const uint64_t g = ((uint64_t)blockIdx.x * NT + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (g >= subtiles) return;
  const uint64_t cw = lay.width / 32, t = g / cw, c0 = (g - t * cw) * 32, c = c0 + lane;
  const uint32_t m = c < lay.n0 ? masks[c * T + t] : 0u;
  const uint64_t off = c < lay.n0 ? offs[c * T + t] : 0ull;
  if constexpr (TROP) {
#pragma unroll 8
    for (int r = 0; r < 32; r++) {
      const uint64_t row = t * 32 + r;
      s_w[warp][r][lane] = row < lay.rows ? D[row * lay.width + c] : WAbs<W>::v;
    }
    __syncwarp();
  }
  uint32_t flags = 0;
  const unsigned lt = (1u << lane) - 1u;
  for (int j = 0; j < 32; j++) {
    const uint32_t mj = __shfl_sync(kFull, m, j);
    const uint64_t oj = __shfl_sync(kFull, off, j);
    if (!((mj >> lane) & 1u)) continue;
    const uint64_t at = oj + __popc(mj & lt);
    if (at >= out_cap) {
      flags |= ST_BOUNDS;
      continue;
    }
    out[at] = (K)(((K)(c0 + j) << lay.b1) | (K)(t * 32 + lane));  // (c0, c1) = (column, row)
    if constexpr (TROP) out_w[at] = s_w[warp][lane][j];
  }
  if (flags) atomicOr(status, flags);
}

// ---- group heads of a Δ sorted by join value ---------------------------------
// A head is the first row of a run of equal join value, or a row at a
// multiple of kGroupMax inside a run; heads whose join value has no edges
// are dropped.  Reduce-then-scan: per-tile (count, degree) sums, one-block
// scans, then the write of (row, degree prefix, segment start, group size).
constexpr int HC_ITEMS = 8;
constexpr uint32_t HC_TILE = NT * HC_ITEMS;

template <class K>
__device__ __forceinline__ uint32_t head_degree(const K* dkeys, uint64_t i, int jshift, uint64_t jmask,
                                                const uint32_t* off, uint64_t n_nodes, uint64_t* jv_out,
                                                uint32_t* full_deg, bool* raw_head = nullptr) {
  const uint64_t jv = ((uint64_t)dkeys[i] >> jshift) & jmask;
  const uint32_t d = jv < n_nodes ? off[jv + 1] - off[jv] : 0u;
  *jv_out = jv;
  *full_deg = d;
  const bool head = (i % kGroupMax) == 0 || (((uint64_t)dkeys[i - 1] >> jshift) & jmask) != jv;
  if (raw_head) *raw_head = head;
  return head ? d : 0u;
}

template <class K>
__global__ void __launch_bounds__(NT)
    k_heads_count(const K* __restrict__ dkeys, uint64_t n, int jshift, uint64_t jmask, const uint32_t* __restrict__ off,
                  uint64_t n_nodes, uint64_t* __restrict__ tile_cnt, uint64_t* __restrict__ tile_deg,
                  unsigned long long* cand_total) {
  __shared__ uint64_t s_red[3][NT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * HC_TILE + (uint64_t)warp * 32 * HC_ITEMS;
  uint64_t c = 0, dsum = 0, cands = 0;
#pragma unroll
  for (int j = 0; j < HC_ITEMS; j++) {
    const uint64_t i = base + (uint64_t)j * 32 + lane;
    if (i < n) {
      uint64_t jv;
      uint32_t fd;
      const uint32_t d = head_degree(dkeys, i, jshift, jmask, off, n_nodes, &jv, &fd);
      c += d ? 1 : 0;
      dsum += d;
      cands += fd;
    }
  }
  c = warp_sum(c);
  dsum = warp_sum(dsum);
  cands = warp_sum(cands);
  if (lane == 0) {
    s_red[0][warp] = c;
    s_red[1][warp] = dsum;
    s_red[2][warp] = cands;
  }
  __syncthreads();
  if (tid == 0) {
    uint64_t a = 0, b = 0, e = 0;
    for (int w = 0; w < NT / 32; w++) {
      a += s_red[0][w];
      b += s_red[1][w];
      e += s_red[2][w];
    }
    tile_cnt[blockIdx.x] = a;
    tile_deg[blockIdx.x] = b;
    if (e) atomicAdd(cand_total, (unsigned long long)e);
  }
}

template <class K>
__global__ void __launch_bounds__(NT)
    k_heads_write(const K* __restrict__ dkeys, uint64_t n, int jshift, uint64_t jmask, const uint32_t* __restrict__ off,
                  uint64_t n_nodes, const uint64_t* __restrict__ tile_cnt, const uint64_t* __restrict__ tile_deg,
                  uint64_t n_tiles, uint32_t* __restrict__ hidx, uint64_t* __restrict__ hpos,
                  uint32_t* __restrict__ hseg, uint8_t* __restrict__ hg) {
  __shared__ uint64_t s_wc[NT / 32], s_wd[NT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * HC_TILE + (uint64_t)warp * 32 * HC_ITEMS;
  uint32_t dg[HC_ITEMS], gs[HC_ITEMS];
  uint64_t exc[HC_ITEMS], exd[HC_ITEMS];
  uint64_t cc = 0, cd = 0;
#pragma unroll
  for (int j = 0; j < HC_ITEMS; j++) {
    const uint64_t i = base + (uint64_t)j * 32 + lane;
    uint32_t d = 0;
    bool rh = false;
    if (i < n) {
      uint64_t jv;
      uint32_t fd;
      d = head_degree(dkeys, i, jshift, jmask, off, n_nodes, &jv, &fd, &rh);
    }
    // The 32 lanes hold one kGroupMax-aligned block of rows, so a group runs
    // from its head to the next head of the block (or the block's end).
    const unsigned hm = __ballot_sync(kFull, rh || i >= n);
    const unsigned above = lane == 31 ? 0u : (hm & (0xffffffffu << (lane + 1)));
    gs[j] = (above ? (uint32_t)(__ffs(above) - 1) : 32u) - (uint32_t)lane;
    dg[j] = d;
    const uint64_t ic = warp_incl_sum((uint64_t)(d ? 1 : 0));
    const uint64_t id = warp_incl_sum((uint64_t)d);
    exc[j] = cc + ic - (d ? 1 : 0);
    exd[j] = cd + id - d;
    cc += __shfl_sync(kFull, ic, 31);
    cd += __shfl_sync(kFull, id, 31);
  }
  if (lane == 0) {
    s_wc[warp] = cc;
    s_wd[warp] = cd;
  }
  __syncthreads();
  uint64_t bc = tile_cnt[blockIdx.x], bd = tile_deg[blockIdx.x];
  for (int w = 0; w < warp; w++) {
    bc += s_wc[w];
    bd += s_wd[w];
  }
#pragma unroll
  for (int j = 0; j < HC_ITEMS; j++) {
    if (!dg[j]) continue;
    const uint64_t i = base + (uint64_t)j * 32 + lane;
    const uint64_t k = bc + exc[j];
    const uint64_t jv = ((uint64_t)dkeys[i] >> jshift) & jmask;
    const uint32_t g = gs[j];
    hidx[k] = (uint32_t)i;
    hpos[k] = bd + exd[j];
    hseg[k] = off[jv];
    hg[k] = (uint8_t)g;
  }
  if (blockIdx.x == gridDim.x - 1 && tid == 0) hpos[tile_cnt[n_tiles]] = tile_deg[n_tiles];
}

// ---- word heads of a Δ held in the marks ------------------------------------
// Two words per thread: a round's marks are a few MB, so small tiles give the
// write (one dependent D-line copy per head word) several waves of blocks.
constexpr int WH_ITEMS = 2;
constexpr uint32_t WH_TILE = NT * WH_ITEMS;
// Rounds after the first keep Δ where the expand left it, in the marks bitmap
// (an entry is in Δ exactly when the round marked it), so Δ needs no key
// compaction: a head is a nonzero marks word whose row (join value
// word / wpr) has edges, and its members are the word's set bits.  Count,
// scan, write as for key heads; the write also snapshots the members'
// merged weights (D → Dprev, which the next expand reads while D changes
// under it) and clears the words for the next round.
template <bool TROP>
__global__ void __launch_bounds__(NT)
    k_words_count(const uint32_t* __restrict__ marks, uint64_t words, uint32_t wpr, const uint32_t* __restrict__ off,
                  uint64_t n_nodes, uint64_t* __restrict__ tile_cnt, uint64_t* __restrict__ tile_deg,
                  unsigned long long* totals) {
  __shared__ uint64_t s_red[4][NT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * WH_TILE + (uint64_t)warp * 32 * WH_ITEMS;
  uint64_t c = 0, dsum = 0, cands = 0, tuples = 0;
#pragma unroll
  for (int j = 0; j < WH_ITEMS; j++) {
    const uint64_t i = base + (uint64_t)j * 32 + lane;
    const uint32_t m = i < words ? marks[i] : 0u;
    if (m) {
      const uint32_t row = (uint32_t)i / wpr;
      const uint32_t d = row < n_nodes ? off[row + 1] - off[row] : 0u;
      const uint32_t pc = __popc(m);
      tuples += pc;
      if (d) {
        c++;
        dsum += d;
        cands += (uint64_t)pc * d;
      }
    }
  }
  c = warp_sum(c);
  dsum = warp_sum(dsum);
  cands = warp_sum(cands);
  tuples = warp_sum(tuples);
  if (lane == 0) {
    s_red[0][warp] = c;
    s_red[1][warp] = dsum;
    s_red[2][warp] = cands;
    s_red[3][warp] = tuples;
  }
  __syncthreads();
  if (tid == 0) {
    uint64_t r[4] = {0, 0, 0, 0};
    for (int w = 0; w < NT / 32; w++)
      for (int q = 0; q < 4; q++) r[q] += s_red[q][w];
    tile_cnt[blockIdx.x] = r[0];
    tile_deg[blockIdx.x] = r[1];
    if (r[2]) atomicAdd(&totals[0], (unsigned long long)r[2]);
    if (r[3]) atomicAdd(&totals[1], (unsigned long long)r[3]);
  }
}

template <bool TROP, class W>
__global__ void __launch_bounds__(NT)
    k_words_write(uint32_t* marks, uint64_t words, uint32_t wpr, const uint32_t* __restrict__ off, uint64_t n_nodes,
                  const uint64_t* __restrict__ tile_cnt, const uint64_t* __restrict__ tile_deg, uint64_t n_tiles,
                  uint32_t* __restrict__ hword, uint32_t* __restrict__ hmask, uint64_t* __restrict__ hpos,
                  uint32_t* __restrict__ hseg, const W* __restrict__ D, W* __restrict__ Dprev,
                  unsigned long long* totals) {
  __shared__ uint64_t s_wc[NT / 32], s_wd[NT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * WH_TILE + (uint64_t)warp * 32 * WH_ITEMS;
  uint32_t mk[WH_ITEMS], dg[WH_ITEMS], sg[WH_ITEMS];
  uint64_t exc[WH_ITEMS], exd[WH_ITEMS];
  uint64_t cc = 0, cd = 0;
#pragma unroll
  for (int j = 0; j < WH_ITEMS; j++) {
    const uint64_t i = base + (uint64_t)j * 32 + lane;
    const uint32_t m = i < words ? marks[i] : 0u;
    uint32_t d = 0, seg = 0;
    if (m) {
      const uint32_t row = (uint32_t)i / wpr;
      if (row < n_nodes) {
        seg = off[row];
        d = off[row + 1] - seg;
      }
      marks[i] = 0u;
    }
    mk[j] = d ? m : 0u;
    dg[j] = d;
    sg[j] = seg;
    const uint64_t ic = warp_incl_sum((uint64_t)(d ? 1 : 0));
    const uint64_t id = warp_incl_sum((uint64_t)d);
    exc[j] = cc + ic - (d ? 1 : 0);
    exd[j] = cd + id - d;
    cc += __shfl_sync(kFull, ic, 31);
    cd += __shfl_sync(kFull, id, 31);
  }
  if (lane == 0) {
    s_wc[warp] = cc;
    s_wd[warp] = cd;
  }
  __syncthreads();
  uint64_t bc = tile_cnt[blockIdx.x], bd = tile_deg[blockIdx.x];
  for (int w = 0; w < warp; w++) {
    bc += s_wc[w];
    bd += s_wd[w];
  }
#pragma unroll
  for (int j = 0; j < WH_ITEMS; j++) {
    const uint64_t i = base + (uint64_t)j * 32 + lane;
    if (dg[j]) {
      const uint64_t k = bc + exc[j];
      hword[k] = (uint32_t)i;
      hmask[k] = mk[j];
      hpos[k] = bd + exd[j];
      hseg[k] = sg[j];
    }
  }
  if constexpr (TROP) {
    // The warp copies the weights of its head words, one 128-byte line per
    // word (one lane per entry; entries outside the mask are copied too and
    // never read), eight lines in flight at a time.
#pragma unroll
    for (int j = 0; j < WH_ITEMS; j++) {
      unsigned hb = __ballot_sync(kFull, dg[j] != 0);
      const uint64_t wb = base + (uint64_t)j * 32;
      while (hb) {
        int t[8];
        W val[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
          t[q] = hb ? __ffs(hb) - 1 : -1;
          hb &= hb - 1;
        }
#pragma unroll
        for (int q = 0; q < 8; q++)
          if (t[q] >= 0) val[q] = D[(wb + t[q]) * 32 + lane];
#pragma unroll
        for (int q = 0; q < 8; q++)
          if (t[q] >= 0) Dprev[(wb + t[q]) * 32 + lane] = val[q];
      }
    }
  }
  if (blockIdx.x == gridDim.x - 1 && tid == 0) {
    hpos[tile_cnt[n_tiles]] = tile_deg[n_tiles];
    totals[2] = tile_cnt[n_tiles];
    totals[3] = tile_deg[n_tiles];
  }
}

inline unsigned grid1(uint64_t n) { return (unsigned)ceil_div(n ? n : 1, NT); }

size_t dense_expand_smem(bool words) {
  return DE_HEADS * (4 + 4 + 4 + (words ? 4 : 1)) + DE_TILE * 2 + kWarps * 32 * kGroupMax * 2 + 16;
}

// (kept, v) → index entry: kept and v are the output key's two columns (which
// one depends on the rule shape), the layout row- or column-major; one of the
// two coefficients is 1, the other the row width.
void out_coefficients(const DenseLayout& lay, int out_pshift, int out_vshift, uint64_t* ck, uint64_t* cv) {
  const bool kept_is_c0 = out_pshift == lay.b1 && out_vshift == 0;
  if (!kept_is_c0 && !(out_pshift == 0 && out_vshift == lay.b1))
    fail(STRATA_E_UNSUPPORTED, "direct-addressed expand: unexpected output key layout");
  const bool kept_is_col = kept_is_c0 == lay.colmajor;  // kept indexes within a row
  *ck = kept_is_col ? 1 : lay.width;
  *cv = kept_is_col ? lay.width : 1;
}

}  // namespace

DenseLayout dense_layout(int b1, uint64_t n0, uint64_t n1, bool colmajor) {
  DenseLayout L{};
  L.b1 = b1;
  L.mask1 = b1 >= 64 ? ~0ull : ((1ull << b1) - 1);
  L.n0 = n0;
  L.n1 = n1;
  L.width = ((colmajor ? n0 : n1) + 31) & ~31ull;
  L.rows = colmajor ? n1 : n0;
  L.entries = L.width * L.rows;
  L.colmajor = colmajor;
  return L;
}

uint64_t dense_tile_size() { return DE_TILE; }
uint32_t dense_group_max() { return kGroupMax; }

template <class K>
void dense_heads(strata_ctx* ctx, const K* dkeys, uint64_t n, int jshift, uint64_t jmask, const uint32_t* off,
                 uint64_t n_nodes, uint64_t* sums, uint32_t* hidx, uint64_t* hpos, uint32_t* hseg, uint8_t* hg,
                 uint64_t* out3) {
  const uint64_t tiles = ceil_div(n ? n : 1, HC_TILE);
  uint64_t* tc = sums;               // tiles + 1
  uint64_t* td = sums + tiles + 1;   // tiles + 1
  uint64_t* ct = sums + 2 * (tiles + 1);
  SK_CUDA(cudaMemsetAsync(ct, 0, 8, ctx->stream));
  k_heads_count<K><<<(unsigned)tiles, NT, 0, ctx->stream>>>(dkeys, n, jshift, jmask, off, n_nodes, tc, td,
                                                            reinterpret_cast<unsigned long long*>(ct));
  after_launch(ctx, "k_heads_count");
  scan_tile_sums(ctx, tc, tiles, 2);  // tc and td
  k_heads_write<K><<<(unsigned)tiles, NT, 0, ctx->stream>>>(dkeys, n, jshift, jmask, off, n_nodes, tc, td, tiles,
                                                            hidx, hpos, hseg, hg);
  after_launch(ctx, "k_heads_write");
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, tc + tiles, 8, cudaMemcpyDeviceToHost, ctx->stream));
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar + 1, td + tiles, 8, cudaMemcpyDeviceToHost, ctx->stream));
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar + 2, ct, 8, cudaMemcpyDeviceToHost, ctx->stream));
  sync_and_check(ctx);
  out3[0] = ctx->h_scalar[0];  // heads
  out3[1] = ctx->h_scalar[1];  // (group, edge) outputs
  out3[2] = ctx->h_scalar[2];  // candidates
}

uint64_t dense_heads_sums(uint64_t n) { return 2 * (ceil_div(n ? n : 1, HC_TILE) + 1) + 2; }

template <class K, bool TROP, class W>
void dense_expand(strata_ctx* ctx, const K* dkeys, const W* dw, uint64_t n_rows, const uint32_t* hidx,
                  const uint64_t* hpos, const uint32_t* hseg, const uint8_t* hg, uint64_t nh, uint64_t total,
                  uint64_t candidates, int pshift, uint64_t pmask, int out_pshift, int out_vshift, const uint32_t* nbr,
                  uint64_t n_nbr, const W* nbr_w, const DenseLayout& lay, uint32_t* bits, W* D,
                  uint32_t* marks, uint64_t* splits_buf) {
  if (nh == 0 || total == 0) return;
  const uint64_t tiles = ceil_div(nh + total, DE_TILE);
  if (tiles > 0x7fffffffull) fail(STRATA_E_UNSUPPORTED, "expand too large for one launch");
  uint64_t ck, cv;
  out_coefficients(lay, out_pshift, out_vshift, &ck, &cv);
  k_tile_splits<<<grid1(tiles + 1), NT, 0, ctx->stream>>>(hpos, nh, total, DE_TILE, tiles, splits_buf);
  after_launch(ctx, "k_tile_splits");
  const int kh = kprof_begin(ctx, K_EXPAND_DENSE);
  const size_t smem = dense_expand_smem(false);
  auto launch = [&](auto kern) {
    SK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<(unsigned)tiles, NT, smem, ctx->stream>>>(dkeys, dw, n_rows, hidx, hpos, hseg, hg, nh, total, splits_buf,
                                                     pshift, pmask, ck, cv, 1u, 0, 33, nbr, n_nbr, nbr_w, lay.entries,
                                                     bits, D, marks, ctx->wshift, ctx->d_status);
  };
  if (lay.entries <= 0xffffffffull) launch(k_expand_dense<K, TROP, false, uint32_t, W>);
  else launch(k_expand_dense<K, TROP, false, uint64_t, W>);
  // Algorithmic bytes: every Δ row (key, weight) once, each head's record,
  // every CSR edge of a group read once (neighbour + weight), one index
  // probe per candidate (a weight for Trop, a 4-byte bitmap word for Bool;
  // a candidate = one Δ row × one edge).
  const uint64_t wsz = TROP ? sizeof(W) : 0;
  kprof_end(ctx, kh, n_rows * (sizeof(K) + wsz) + nh * (4 + 8 + 4 + 1) + total * (4 + wsz) +
                         candidates * (TROP ? sizeof(W) : 4));
  after_launch(ctx, "k_expand_dense");
}

template <bool TROP, class W>
void dense_word_heads(strata_ctx* ctx, uint32_t* marks, const DenseLayout& lay, const uint32_t* off,
                      uint64_t n_nodes, uint64_t* sums, uint32_t* hword, uint32_t* hmask, uint64_t* hpos,
                      uint32_t* hseg, const W* D, W* Dprev, uint64_t* out4) {
  const uint64_t words = lay.entries / 32;
  if (words >= (1ull << 32)) fail(STRATA_E_UNSUPPORTED, "direct-addressed index beyond 2^37 entries");
  const uint64_t tiles = ceil_div(words ? words : 1, WH_TILE);
  uint64_t* tc = sums;
  uint64_t* td = sums + tiles + 1;
  auto* tot = reinterpret_cast<unsigned long long*>(sums + 2 * (tiles + 1));
  SK_CUDA(cudaMemsetAsync(tot, 0, 4 * 8, ctx->stream));
  const uint32_t wpr = (uint32_t)(lay.width / 32);
  k_words_count<TROP><<<(unsigned)tiles, NT, 0, ctx->stream>>>(marks, words, wpr, off, n_nodes, tc, td, tot);
  after_launch(ctx, "k_words_count");
  scan_tile_sums(ctx, tc, tiles, 2);  // tc and td
  k_words_write<TROP, W><<<(unsigned)tiles, NT, 0, ctx->stream>>>(marks, words, wpr, off, n_nodes, tc, td, tiles,
                                                                  hword, hmask, hpos, hseg, D, Dprev, tot);
  after_launch(ctx, "k_words_write");
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, tot, 4 * 8, cudaMemcpyDeviceToHost, ctx->stream));
  sync_and_check(ctx);
  out4[0] = ctx->h_scalar[2];  // heads
  out4[1] = ctx->h_scalar[3];  // (head, edge) outputs
  out4[2] = ctx->h_scalar[0];  // candidates
  out4[3] = ctx->h_scalar[1];  // Δ tuples
}

uint64_t dense_word_heads_sums(const DenseLayout& lay) { return 2 * (ceil_div(lay.entries / 32 + 1, WH_TILE) + 1) + 4; }

template <bool TROP, class W>
void dense_expand_words(strata_ctx* ctx, const uint32_t* hword, const uint32_t* hmask, const uint64_t* hpos,
                        const uint32_t* hseg, uint64_t nh, uint64_t total, uint64_t candidates, uint64_t n_delta,
                        const W* Dprev, int out_pshift, int out_vshift, const uint32_t* nbr, uint64_t n_nbr,
                        const W* nbr_w, const DenseLayout& lay, uint32_t* bits, W* D, uint32_t* marks,
                        uint64_t* splits_buf) {
  if (nh == 0 || total == 0) return;
  const uint64_t tiles = ceil_div(nh + total, DE_TILE);
  if (tiles > 0x7fffffffull) fail(STRATA_E_UNSUPPORTED, "expand too large for one launch");
  uint64_t ck, cv;
  out_coefficients(lay, out_pshift, out_vshift, &ck, &cv);
  k_tile_splits<<<grid1(tiles + 1), NT, 0, ctx->stream>>>(hpos, nh, total, DE_TILE, tiles, splits_buf);
  after_launch(ctx, "k_tile_splits");
  const int kh = kprof_begin(ctx, K_EXPAND_DENSE);
  const size_t smem = dense_expand_smem(true);
  const uint32_t wpr = (uint32_t)(lay.width / 32);
  const int wpr_shift = (wpr & (wpr - 1)) == 0 ? __builtin_ctz(wpr) : -1;
  const int members = ctx->tune_dense_members ? ctx->tune_dense_members : kDenseMembers;
  auto launch = [&](auto kern) {
    SK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<(unsigned)tiles, NT, smem, ctx->stream>>>(nullptr, Dprev, lay.entries, hword, hpos, hseg, hmask, nh, total,
                                                     splits_buf, 0, 0, ck, cv, wpr, wpr_shift, members, nbr, n_nbr,
                                                     nbr_w, lay.entries, bits, D, marks, ctx->wshift, ctx->d_status);
  };
  if (lay.entries <= 0xffffffffull) launch(k_expand_dense<uint32_t, TROP, true, uint32_t, W>);
  else launch(k_expand_dense<uint32_t, TROP, true, uint64_t, W>);
  // Algorithmic bytes: each head's record (word, mask, position, segment),
  // every CSR edge of a head read once (neighbour + weight), each Δ weight
  // once, one index probe per candidate (a weight for Trop, a 4-byte bitmap
  // word for Bool).
  const uint64_t wsz = TROP ? sizeof(W) : 0;
  kprof_end(ctx, kh, nh * (4 + 4 + 8 + 4) + total * (4 + wsz) + n_delta * wsz + candidates * (TROP ? sizeof(W) : 4));
  after_launch(ctx, "k_expand_dense");
}

template <class K, bool TROP, class W>
uint64_t dense_marks_compact(strata_ctx* ctx, uint32_t* marks, const DenseLayout& lay, const W* D, K* out,
                             W* out_w, uint64_t out_cap, uint64_t* sums) {
  const uint64_t words = (lay.entries + 31) / 32;
  const uint64_t tiles = ceil_div(words, MC_TILE);
  k_marks_count<<<(unsigned)tiles, NT, 0, ctx->stream>>>(marks, words, sums);
  after_launch(ctx, "k_marks_count");
  scan_tile_sums(ctx, sums, tiles);
  k_marks_write<K, TROP, W><<<(unsigned)tiles, NT, 0, ctx->stream>>>(marks, words, lay, D, out, out_w, out_cap,
                                                                    sums, ctx->d_status);
  after_launch(ctx, "k_marks_write");
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, sums + tiles, 8, cudaMemcpyDeviceToHost, ctx->stream));
  sync_and_check(ctx);
  return ctx->h_scalar[0];
}

uint64_t dense_marks_states(uint64_t entries) { return ceil_div((entries + 31) / 32, MC_TILE) + 2; }

template <class K, bool TROP, class W>
void dense_seed(strata_ctx* ctx, const K* keys, const W* w, uint64_t n, const DenseLayout& lay, uint32_t* bits,
                W* D, uint32_t* marks) {
  if (TROP) {
    k_fill_w<W><<<(unsigned)std::min<uint64_t>(ceil_div(lay.entries, NT), (uint64_t)ctx->num_sms * 16), NT, 0,
                  ctx->stream>>>(D, lay.entries, WAbs<W>::v);
    after_launch(ctx, "k_fill_w");
  }
  if (!n) return;
  k_dense_seed<K, TROP, W><<<grid1(n), NT, 0, ctx->stream>>>(keys, w, n, lay, bits, D, marks, ctx->d_status);
  after_launch(ctx, "k_dense_seed");
}

template <class K, bool TROP, class W>
uint64_t dense_compact(strata_ctx* ctx, const uint32_t* bits, const W* D, const DenseLayout& lay, K* out,
                       W* out_w, uint64_t out_cap) {
  const uint64_t logical = lay.n0 * lay.n1;
  if (!logical) return 0;
  if (lay.colmajor) {
    const uint64_t T = ceil_div(lay.rows, 32), subtiles = T * (lay.width / 32), M = lay.n0 * T;
    const uint64_t chunks = ceil_div(M, CM_CHUNK);
    const unsigned blocks = (unsigned)ceil_div(subtiles, NT / 32);
    DBuf<uint32_t> masks(ctx, M);
    DBuf<uint64_t> offs(ctx, M), sums(ctx, chunks + 1);
    k_cm_masks<TROP, W><<<blocks, NT, 0, ctx->stream>>>(bits, D, lay, T, subtiles, masks.p);
    after_launch(ctx, "k_cm_masks");
    k_cm_chunk_sums<<<(unsigned)chunks, NT, 0, ctx->stream>>>(masks.p, M, sums.p);
    after_launch(ctx, "k_cm_chunk_sums");
    scan_tile_sums(ctx, sums.p, chunks);
    k_cm_offsets<<<(unsigned)chunks, NT, 0, ctx->stream>>>(masks.p, M, sums.p, offs.p);
    after_launch(ctx, "k_cm_offsets");
    const size_t smem = TROP ? cm_write_smem<W>() : 0;
    if (smem > 48 * 1024)
      SK_CUDA(cudaFuncSetAttribute(k_cm_write<K, TROP, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_cm_write<K, TROP, W><<<blocks, NT, smem, ctx->stream>>>(bits, D, lay, T, subtiles, masks.p, offs.p, out, out_w,
                                                               out_cap, ctx->d_status);
    after_launch(ctx, "k_cm_write");
    SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, sums.p + chunks, 8, cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
    return ctx->h_scalar[0];
  }
  const uint64_t tiles = ceil_div(logical, DC_TILE);
  DBuf<uint64_t> states(ctx, tiles + 2);
  uint32_t* counter = reinterpret_cast<uint32_t*>(states.p + tiles + 1);
  SK_CUDA(cudaMemsetAsync(states.p, 0, sizeof(uint64_t) * (tiles + 2), ctx->stream));
  k_dense_compact<K, TROP, W><<<(unsigned)tiles, NT, 0, ctx->stream>>>(bits, D, lay, out, out_w, out_cap, states.p,
                                                                       counter, states.p + tiles, ctx->d_status);
  after_launch(ctx, "k_dense_compact");
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, states.p + tiles, 8, cudaMemcpyDeviceToHost, ctx->stream));
  sync_and_check(ctx);
  return ctx->h_scalar[0];
}

#define SK_INST_DENSE(K, T, W)                                                                              \
  template void dense_expand<K, T, W>(strata_ctx*, const K*, const W*, uint64_t, const uint32_t*, const uint64_t*, \
                                      const uint32_t*, const uint8_t*, uint64_t, uint64_t, uint64_t, int, uint64_t, \
                                      int, int, const uint32_t*, uint64_t, const W*, const DenseLayout&, uint32_t*, \
                                      W*, uint32_t*, uint64_t*);                                                  \
  template uint64_t dense_marks_compact<K, T, W>(strata_ctx*, uint32_t*, const DenseLayout&, const W*, K*, W*,     \
                                                 uint64_t, uint64_t*);                                            \
  template void dense_seed<K, T, W>(strata_ctx*, const K*, const W*, uint64_t, const DenseLayout&, uint32_t*, W*, \
                                    uint32_t*);                                                                   \
  template uint64_t dense_compact<K, T, W>(strata_ctx*, const uint32_t*, const W*, const DenseLayout&, K*, W*,     \
                                           uint64_t);
template void dense_heads<uint32_t>(strata_ctx*, const uint32_t*, uint64_t, int, uint64_t, const uint32_t*, uint64_t,
                                    uint64_t*, uint32_t*, uint64_t*, uint32_t*, uint8_t*, uint64_t*);
template void dense_heads<uint64_t>(strata_ctx*, const uint64_t*, uint64_t, int, uint64_t, const uint32_t*, uint64_t,
                                    uint64_t*, uint32_t*, uint64_t*, uint32_t*, uint8_t*, uint64_t*);
SK_INST_DENSE(uint32_t, false, int32_t)
SK_INST_DENSE(uint32_t, true, int32_t)
SK_INST_DENSE(uint32_t, true, int64_t)
SK_INST_DENSE(uint64_t, false, int32_t)
SK_INST_DENSE(uint64_t, true, int32_t)
SK_INST_DENSE(uint64_t, true, int64_t)
#undef SK_INST_DENSE
#define SK_INST_WORDS(T, W)                                                                                     \
  template void dense_word_heads<T, W>(strata_ctx*, uint32_t*, const DenseLayout&, const uint32_t*, uint64_t,   \
                                       uint64_t*, uint32_t*, uint32_t*, uint64_t*, uint32_t*, const W*, W*,     \
                                       uint64_t*);                                                              \
  template void dense_expand_words<T, W>(strata_ctx*, const uint32_t*, const uint32_t*, const uint64_t*,        \
                                         const uint32_t*, uint64_t, uint64_t, uint64_t, uint64_t, const W*, int, \
                                         int, const uint32_t*, uint64_t, const W*, const DenseLayout&,          \
                                         uint32_t*, W*, uint32_t*, uint64_t*);
SK_INST_WORDS(false, int32_t)
SK_INST_WORDS(true, int32_t)
SK_INST_WORDS(true, int64_t)
#undef SK_INST_WORDS

}  // namespace sk
