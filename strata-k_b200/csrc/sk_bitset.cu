// sk_bitset.cu — bit-parallel semi-naive transitive closure, one instance or
// a batch of independent instances.
//
// The program is   path(X,Y) :- edge(X,Y).   path(X,Z) :- edge(X,Y), path(Y,Z).
// evaluated semi-naively exactly as the interpreter does
// (strata-eval/src/seminaive.rs:29-106, 192-209): the bootstrap round derives
// Δ0 = edge, then every round derives
//     Δ'(X, ·) = ( ∪_{Y ∈ out(X)} Δ(Y, ·) ) ∖ path(X, ·),   path ∪= Δ'
// until Δ' is empty.  Here each relation row is a bit row over the Z domain,
// so one OR of a 128-bit word joins 128 Δ tuples at once, the AND-NOT is the
// dedup and Δ-difference, and the popcount of the new bits is |Δ'|.  Rounds,
// Δ sets and the final relation are those of the tuple plans.
//
// Layout (per instance i): rows X ∈ [0, n_rows), each row W4 = ceil(n_cols /
// 128) uint4 words; three matrices (path F, Δ and Δ' double-buffered) plus a
// byte flag per row (Δ row non-empty) and an out-edge CSR with local ids.
// All instances of a wave share one pool; instance i starts at vec_base[i]
// and row_base[i].
//
// Work split.  A unit is one warp over (32 / L) consecutive rows of one
// instance, L = min(32, next power of two >= W4) lanes per row, so a
// 100-node instance packs 32 rows into a warp and a 50,000-node instance
// gives each row a whole warp.  Per round one persistent kernel strides its
// warps over the units of all active instances of the wave (the unit prefix
// over active instances is rebuilt on the device by a one-block bookkeeping
// kernel after each round), and the host replays a captured CUDA graph of R
// (round, bookkeeping) pairs until no instance is active — one launch per
// semi-naive round for the whole batch, no host round trip inside the graph.
//
// Summary per instance: |path| and  fp = Σ_{(X,Z) ∈ path} mix64(X) · c^Z
// (mod 2^64, c = 0x9E3779B97F4A7C15), computed from the bit rows one 32-bit
// word at a time with byte tables.
#include "sk_ops.cuh"
#include "sk_prims.cuh"
#include "sk_rel.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace sk {
namespace {

constexpr int BS_NT = 256;
constexpr uint64_t kPolyC = 0x9e3779b97f4a7c15ull;

// Device view of a wave (all pointers into fixed buffers of the call).
struct BsView {
  // per instance of the wave
  const uint32_t* n_rows;
  const uint32_t* n_cols;
  const uint32_t* w4;
  const uint8_t* lshift;  // log2(lanes per row)
  const uint64_t* row_base;
  const uint64_t* vec_base;
  uint64_t* delta;   // |Δ'| of the current round
  uint64_t* total;   // |path| so far
  uint32_t* rounds;
  uint8_t* active;
  // active list and unit prefix (rebuilt by k_bs_book)
  uint32_t* act;
  uint64_t* uprefix;
  uint32_t* n_act;
  uint64_t* u_total;
  // CSR over global rows, local neighbour ids
  const uint64_t* off;
  const uint32_t* nbr;
  // matrices and row flags
  uint4* F;
  uint4* D0;
  uint4* D1;
  uint8_t* f0;
  uint8_t* f1;
  unsigned long long* bytes;  // algorithmic bytes of the rounds (profiling), or null
  uint32_t* status;
};

__device__ __forceinline__ uint32_t popc4(const uint4& a) {
  return __popc(a.x) + __popc(a.y) + __popc(a.z) + __popc(a.w);
}
__device__ __forceinline__ bool any4(const uint4& a) { return (a.x | a.y | a.z | a.w) != 0u; }

// Instance slot k of unit u: uprefix[k] <= u < uprefix[k + 1].
__device__ __forceinline__ uint32_t unit_owner(const uint64_t* uprefix, uint32_t n, uint64_t u) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (uprefix[mid] <= u) lo = mid; else hi = mid;
  }
  return lo;
}

// One semi-naive round over every active instance of the wave.  Reads Δ from
// (D_PAR, f_PAR), writes Δ' to the other buffer pair and updates F.
template <int PAR>
__global__ void __launch_bounds__(BS_NT) k_bs_round(BsView v) {
  const uint32_t n_act = *v.n_act;
  const uint64_t U = *v.u_total;
  const uint4* __restrict__ Dc = PAR ? v.D1 : v.D0;
  uint4* __restrict__ Dn = PAR ? v.D0 : v.D1;
  const uint8_t* __restrict__ fc = PAR ? v.f1 : v.f0;
  uint8_t* __restrict__ fn = PAR ? v.f0 : v.f1;
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = (uint64_t)gridDim.x * (BS_NT / 32);
  unsigned long long moved = 0;
  for (uint64_t u = ((uint64_t)blockIdx.x * BS_NT + threadIdx.x) >> 5; u < U; u += nwarps) {
    const uint32_t k = unit_owner(v.uprefix, n_act, u);
    const uint32_t i = v.act[k];
    const uint32_t n = v.n_rows[i], W = v.w4[i];
    const int ls = v.lshift[i];
    const uint32_t lpr = 1u << ls, sub = (uint32_t)lane >> ls, sl = (uint32_t)lane & (lpr - 1);
    const unsigned smask = ls == 5 ? 0xffffffffu : (((1u << lpr) - 1u) << (sub << ls));
    const uint64_t X = (u - v.uprefix[k]) * (32u >> ls) + sub;
    const bool valid = X < n;
    const uint64_t rb = v.row_base[i], vb = v.vec_base[i];
    const uint64_t e0 = valid ? v.off[rb + X] : 0, e1 = valid ? v.off[rb + X + 1] : 0;
    // Does the row join any non-empty Δ row?
    bool any_y = false;
    for (uint64_t e = e0 + sl; e < e1; e += lpr) {
      const uint32_t y = v.nbr[e];
      if (y < n && fc[rb + y]) any_y = true;
    }
    // every lane takes part in the ballot (lanes past the last row included)
    const unsigned bal_y = __ballot_sync(kFull, any_y);
    const bool row_has = valid && (bal_y & smask) != 0u;
    bool row_any = false;
    uint32_t cnt = 0;
    if (row_has) {
      uint32_t active_edges = 0, acc_words = 0;
      for (uint32_t c = sl; c < W; c += lpr) {
        uint4 acc = make_uint4(0u, 0u, 0u, 0u);
        active_edges = 0;
        // four edges at a time: their neighbour, flag and Δ-row loads are
        // independent, so they are in flight together
        for (uint64_t e = e0; e < e1; e += 4) {
          uint32_t y[4];
          bool on[4];
#pragma unroll
          for (int q = 0; q < 4; q++) y[q] = e + q < e1 ? v.nbr[e + q] : 0xffffffffu;
#pragma unroll
          for (int q = 0; q < 4; q++) on[q] = y[q] < n && fc[rb + y[q]] != 0;
          uint4 d[4];
#pragma unroll
          for (int q = 0; q < 4; q++) d[q] = on[q] ? Dc[vb + (uint64_t)y[q] * W + c] : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
          for (int q = 0; q < 4; q++) {
            acc.x |= d[q].x;
            acc.y |= d[q].y;
            acc.z |= d[q].z;
            acc.w |= d[q].w;
            active_edges += on[q] ? 1u : 0u;
          }
        }
        uint4 nw = make_uint4(0u, 0u, 0u, 0u);
        if (any4(acc)) {
          acc_words++;
          uint4* fp = v.F + vb + X * W + c;
          uint4 f = *fp;
          nw = make_uint4(acc.x & ~f.x, acc.y & ~f.y, acc.z & ~f.z, acc.w & ~f.w);
          if (any4(nw)) {
            f = make_uint4(f.x | nw.x, f.y | nw.y, f.z | nw.z, f.w | nw.w);
            *fp = f;
            cnt += popc4(nw);
            row_any = true;
          }
        }
        Dn[vb + X * W + c] = nw;
      }
      if (v.bytes) {
        // this lane's words: Δ rows read, Δ' written, path read (and written
        // where bits are new); its share of the edge list and flags
        const uint64_t lw = (W > sl) ? (W - sl + lpr - 1) / lpr : 0;
        moved += lw * 16ull * (active_edges + 1) + acc_words * 32ull + (sl == 0 ? (e1 - e0) * 5ull : 0ull);
      }
    }
    const unsigned bal = __ballot_sync(kFull, row_any);
    if (valid && sl == 0) fn[rb + X] = (bal & smask) != 0u ? 1 : 0;
    cnt = warp_sum(cnt);
    if (lane == 0 && cnt) atomicAdd(reinterpret_cast<unsigned long long*>(&v.delta[i]), (unsigned long long)cnt);
  }
  if (v.bytes) {
    moved = warp_sum(moved);
    if (lane == 0 && moved) atomicAdd(v.bytes, moved);
  }
}

// After a round (or the bootstrap): close finished instances, add |Δ'| to
// |path|, rebuild the active list and its unit prefix.  One block.
constexpr int BK_NT = 1024;
__global__ void __launch_bounds__(BK_NT) k_bs_book(BsView v, uint32_t n_inst, int count_round) {
  __shared__ uint64_t s_scan[BK_NT / 32 + 1];
  __shared__ uint64_t s_carry[2];
  if (threadIdx.x == 0) s_carry[0] = s_carry[1] = 0;
  __syncthreads();
  for (uint32_t base = 0; base < n_inst; base += BK_NT) {
    const uint32_t i = base + threadIdx.x;
    uint64_t units = 0, act = 0;
    if (i < n_inst && v.active[i]) {
      const uint64_t d = v.delta[i];
      v.delta[i] = 0;
      if (count_round) v.rounds[i]++;
      if (d == 0) {
        v.active[i] = 0;
      } else {
        v.total[i] += d;
        act = 1;
        const uint32_t rpu = 32u >> v.lshift[i];
        units = (v.n_rows[i] + rpu - 1) / rpu;
      }
    }
    uint64_t tot_a, tot_u;
    const uint64_t ex_a = block_excl_sum<BK_NT>(act, s_scan, &tot_a);
    __syncthreads();
    const uint64_t ex_u = block_excl_sum<BK_NT>(units, s_scan, &tot_u);
    if (act) {
      v.act[s_carry[0] + ex_a] = i;
      v.uprefix[s_carry[0] + ex_a] = s_carry[1] + ex_u;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      s_carry[0] += tot_a;
      s_carry[1] += tot_u;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    v.uprefix[s_carry[0]] = s_carry[1];
    *v.n_act = (uint32_t)s_carry[0];
    *v.u_total = s_carry[1];
  }
}

// Instance of a wave-local edge index (edge offsets relative to the wave).
__device__ __forceinline__ uint32_t edge_owner(const uint64_t* eoff, uint32_t n_inst, uint64_t g) {
  uint32_t lo = 0, hi = n_inst;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (eoff[mid] <= g) lo = mid; else hi = mid;
  }
  return lo;
}

// Out-degree per global row.
__global__ void k_bs_degree(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, uint64_t m,
                            const uint64_t* __restrict__ eoff, uint32_t n_inst, BsView v, uint32_t* deg,
                            uint32_t* bad) {
  for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < m; g += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t i = edge_owner(eoff, n_inst, g);
    const uint32_t x = src[g], y = dst[g];
    if (x >= v.n_rows[i] || y >= v.n_cols[i]) {
      *bad = 1u;  // an edge endpoint outside its instance's nodes
      continue;
    }
    atomicAdd(&deg[v.row_base[i] + x], 1u);
  }
}

// Exclusive scan of u32 degrees into u64 offsets: per-tile sums, one-block
// scan of the sums, then the write.
constexpr uint32_t SC_TILE = 2048;
__global__ void __launch_bounds__(BS_NT) k_bs_tile_sums(const uint32_t* __restrict__ deg, uint64_t n,
                                                        uint64_t* __restrict__ sums) {
  __shared__ uint64_t s_red[BS_NT / 32];
  uint64_t s = 0;
  const uint64_t b = (uint64_t)blockIdx.x * SC_TILE;
  for (uint32_t j = threadIdx.x; j < SC_TILE; j += BS_NT)
    if (b + j < n) s += deg[b + j];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t t = 0;
    for (int w = 0; w < BS_NT / 32; w++) t += s_red[w];
    sums[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(BS_NT) k_bs_tile_write(const uint32_t* __restrict__ deg, uint64_t n,
                                                         const uint64_t* __restrict__ sums, uint64_t* __restrict__ off,
                                                         uint64_t* __restrict__ cursor) {
  __shared__ uint64_t s_scan[BS_NT / 32 + 1];
  __shared__ uint64_t s_carry;
  if (threadIdx.x == 0) s_carry = sums[blockIdx.x];
  __syncthreads();
  const uint64_t b = (uint64_t)blockIdx.x * SC_TILE;
  for (uint32_t j0 = 0; j0 < SC_TILE; j0 += BS_NT) {
    const uint64_t r = b + j0 + threadIdx.x;
    const uint64_t d = r < n ? deg[r] : 0;
    uint64_t tot;
    const uint64_t ex = block_excl_sum<BS_NT>(d, s_scan, &tot);
    if (r < n) {
      off[r] = s_carry + ex;
      cursor[r] = s_carry + ex;
    }
    __syncthreads();
    if (threadIdx.x == 0) s_carry += tot;
    __syncthreads();
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) off[n] = s_carry;
}

// Scatter edges into the CSR (order within a row is free: the round ORs) and
// seed path = Δ0 = edge bits, counting distinct edges per instance.
__global__ void k_bs_seed(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, uint64_t m,
                          const uint64_t* __restrict__ eoff, uint32_t n_inst, BsView v, uint64_t* cursor,
                          uint32_t* nbr) {
  const int lane = threadIdx.x & 31;
  for (uint64_t g0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~31ull; g0 < m;
       g0 += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t g = g0 + lane;
    uint32_t fresh = 0, i = 0xffffffffu;
    if (g < m) {
      i = edge_owner(eoff, n_inst, g);
      const uint32_t x = src[g], y = dst[g];
      if (x < v.n_rows[i] && y < v.n_cols[i]) {
        const uint64_t row = v.row_base[i] + x;
        nbr[atomicAdd(reinterpret_cast<unsigned long long*>(&cursor[row]), 1ull)] = y;
        uint32_t* Fw = reinterpret_cast<uint32_t*>(v.F + v.vec_base[i] + (uint64_t)x * v.w4[i]);
        const uint32_t bit = 1u << (y & 31);
        const uint32_t old = atomicOr(&Fw[y >> 5], bit);
        fresh = (old & bit) ? 0u : 1u;
      }
    }
    // per-instance distinct-edge counts (warp-aggregated when the warp is one instance)
    const uint32_t i0 = __shfl_sync(kFull, i, 0);
    if (__all_sync(kFull, i == i0 || i == 0xffffffffu)) {
      const uint32_t c = warp_sum(fresh);
      if (lane == 0 && c && i0 != 0xffffffffu)
        atomicAdd(reinterpret_cast<unsigned long long*>(&v.delta[i0]), (unsigned long long)c);
    } else if (fresh) {
      atomicAdd(reinterpret_cast<unsigned long long*>(&v.delta[i]), 1ull);
    }
  }
}

// Δ0 row flags: a row of path0 is non-empty iff the node has out-edges.
__global__ void k_bs_flags0(const uint64_t* __restrict__ off, uint64_t rows, uint8_t* f0) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x)
    f0[r] = off[r + 1] > off[r] ? 1 : 0;
}

// |path| and Σ mix64(X) · c^Z per instance from the final bit rows.
// tpw[w] = c^(32 w); tables tb[b][v] = Σ_{j ∈ bits(v)} c^(8 b + j).
__global__ void __launch_bounds__(BS_NT) k_bs_final(BsView v, const uint64_t* __restrict__ tpw,
                                                    const uint64_t* __restrict__ tb_g, uint64_t* counts,
                                                    uint64_t* fps) {
  __shared__ uint64_t tb[4][256];
  for (int t = threadIdx.x; t < 1024; t += BS_NT) (&tb[0][0])[t] = tb_g[t];
  __syncthreads();
  const uint32_t n_act = *v.n_act;
  const uint64_t U = *v.u_total;
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = (uint64_t)gridDim.x * (BS_NT / 32);
  for (uint64_t u = ((uint64_t)blockIdx.x * BS_NT + threadIdx.x) >> 5; u < U; u += nwarps) {
    const uint32_t k = unit_owner(v.uprefix, n_act, u);
    const uint32_t i = v.act[k];
    const uint32_t n = v.n_rows[i], W = v.w4[i];
    const int ls = v.lshift[i];
    const uint32_t lpr = 1u << ls, sub = (uint32_t)lane >> ls, sl = (uint32_t)lane & (lpr - 1);
    const uint64_t X = (u - v.uprefix[k]) * (32u >> ls) + sub;
    uint64_t cnt = 0, poly = 0;
    if (X < n) {
      const uint4* row = v.F + v.vec_base[i] + X * W;
      for (uint32_t c = sl; c < W; c += lpr) {
        const uint4 q = row[c];
        const uint32_t wd[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int h = 0; h < 4; h++) {
          const uint32_t x = wd[h];
          if (!x) continue;
          cnt += __popc(x);
          const uint64_t t = tb[0][x & 255] + tb[1][(x >> 8) & 255] + tb[2][(x >> 16) & 255] + tb[3][x >> 24];
          poly += tpw[4 * (uint64_t)c + h] * t;
        }
      }
      // splitmix64 finalizer of X
      uint64_t z = X + kPolyC;
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
      z ^= z >> 31;
      poly *= z;
    }
    cnt = warp_sum(cnt);
    poly = warp_sum(poly);
    if (lane == 0) {
      if (cnt) atomicAdd(reinterpret_cast<unsigned long long*>(&counts[i]), (unsigned long long)cnt);
      if (poly) atomicAdd(reinterpret_cast<unsigned long long*>(&fps[i]), (unsigned long long)poly);
    }
  }
}

inline uint32_t lanes_shift(uint32_t w4) {
  int s = 0;
  while (s < 5 && (1u << s) < w4) s++;
  return (uint32_t)s;
}

// Fixed buffers of one call, sized for the largest wave.
struct BsBuffers {
  DBuf<uint32_t> n_rows, n_cols, w4, act, n_act, deg, bad;
  DBuf<uint8_t> lshift, active, f0, f1;
  DBuf<uint64_t> row_base, vec_base, delta, total, uprefix, u_total, off, cursor, eoff, sums, bytes;
  DBuf<uint32_t> rounds, nbr;
  DBuf<uint4> F, D0, D1;
  explicit BsBuffers(strata_ctx* c) {
    for (auto* b : {&n_rows, &n_cols, &w4, &act, &n_act, &deg, &bad, &rounds, &nbr}) b->ctx = c;
    for (auto* b : {&lshift, &active, &f0, &f1}) b->ctx = c;
    for (auto* b : {&row_base, &vec_base, &delta, &total, &uprefix, &u_total, &off, &cursor, &eoff, &sums, &bytes})
      b->ctx = c;
    F.ctx = D0.ctx = D1.ctx = c;
  }
  BsView view(bool profile) {
    BsView v;
    v.n_rows = n_rows.p;
    v.n_cols = n_cols.p;
    v.w4 = w4.p;
    v.lshift = lshift.p;
    v.row_base = row_base.p;
    v.vec_base = vec_base.p;
    v.delta = delta.p;
    v.total = total.p;
    v.rounds = rounds.p;
    v.active = active.p;
    v.act = act.p;
    v.uprefix = uprefix.p;
    v.n_act = n_act.p;
    v.u_total = u_total.p;
    v.off = off.p;
    v.nbr = nbr.p;
    v.F = F.p;
    v.D0 = D0.p;
    v.D1 = D1.p;
    v.f0 = f0.p;
    v.f1 = f1.p;
    v.bytes = profile ? reinterpret_cast<unsigned long long*>(bytes.p) : nullptr;
    v.status = nullptr;
    return v;
  }
};

struct InstSpec {
  uint32_t rows, cols;
  uint64_t e0, e1;  // edge range in the input arrays
};

inline uint64_t inst_w4(const InstSpec& s) { return std::max<uint64_t>(1, ceil_div(s.cols, 128)); }
inline uint64_t inst_vecs(const InstSpec& s) { return (uint64_t)s.rows * inst_w4(s); }
inline uint64_t inst_bytes(const InstSpec& s) {
  return 3 * inst_vecs(s) * 16 + (uint64_t)s.rows * (2 + 4 + 16) + (s.e1 - s.e0) * 4 + 64;
}

struct BsResult {
  std::vector<uint64_t> counts, fps, totals;
  std::vector<uint32_t> rounds;
  uint64_t waves = 0, graph_launches = 0, round_launches = 0, bytes = 0;
  uint32_t rounds_max = 0;
};

// Host tables of the fingerprint: c^(32 w) for w < words, and the byte tables.
void poly_tables(uint64_t words, std::vector<uint64_t>& tpw, std::vector<uint64_t>& tb) {
  tpw.resize(std::max<uint64_t>(words, 1));
  uint64_t c32 = 1;
  for (int j = 0; j < 32; j++) c32 *= kPolyC;
  uint64_t a = 1;
  for (uint64_t w = 0; w < tpw.size(); w++) {
    tpw[w] = a;
    a *= c32;
  }
  uint64_t pw[32];
  pw[0] = 1;
  for (int j = 1; j < 32; j++) pw[j] = pw[j - 1] * kPolyC;
  tb.assign(1024, 0);
  for (int b = 0; b < 4; b++)
    for (int x = 0; x < 256; x++) {
      uint64_t s = 0;
      for (int j = 0; j < 8; j++)
        if (x >> j & 1) s += pw[8 * b + j];
      tb[b * 256 + x] = s;
    }
}

int round_grid(strata_ctx* ctx) {
  int per_sm = 0;
  check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bs_round<0>, BS_NT, 0), "occupancy");
  if (ctx->tune_bs_blocks > 0) per_sm = std::min(per_sm, ctx->tune_bs_blocks);
  return std::max(1, per_sm) * ctx->num_sms;
}

// Run instances `order[lo..hi)` as waves within `budget` bytes (mode 0:
// graph-replayed batched rounds; mode 1: one instance per launch, host-driven
// rounds).  When `keep_bits` is set (a single instance) F is left in `bufs`.
void bs_run(strata_ctx* ctx, const std::vector<InstSpec>& spec, const uint32_t* d_src, const uint32_t* d_dst,
            int mode, uint64_t budget, BsBuffers& B, BsResult& R, bool want_fp) {
  const uint32_t n_inst = (uint32_t)spec.size();
  R.counts.assign(n_inst, 0);
  R.fps.assign(n_inst, 0);
  R.totals.assign(n_inst, 0);
  R.rounds.assign(n_inst, 0);
  // order: largest first (mode 0 packs waves; mode 1 runs one at a time)
  std::vector<uint32_t> order(n_inst);
  for (uint32_t i = 0; i < n_inst; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return inst_vecs(spec[a]) > inst_vecs(spec[b]); });
  std::vector<std::pair<uint32_t, uint32_t>> waves;  // ranges of `order`
  {
    uint32_t a = 0;
    while (a < n_inst) {
      uint64_t bytes = inst_bytes(spec[order[a]]);
      if (bytes > budget) fail(STRATA_E_OOM, "one instance's bit matrices exceed the memory budget");
      uint32_t b = a + 1;
      if (mode == 0)
        while (b < n_inst && bytes + inst_bytes(spec[order[b]]) <= budget) bytes += inst_bytes(spec[order[b]]), b++;
      waves.push_back({a, b});
      a = b;
    }
  }
  // size the fixed buffers for the largest wave
  uint64_t max_rows = 1, max_vecs = 1, max_edges = 1, max_w32 = 1;
  uint32_t max_n = 1;
  for (auto& w : waves) {
    uint64_t rows = 0, vecs = 0, edges = 0;
    for (uint32_t k = w.first; k < w.second; k++) {
      const InstSpec& s = spec[order[k]];
      rows += s.rows;
      vecs += inst_vecs(s);
      edges += s.e1 - s.e0;
      max_w32 = std::max<uint64_t>(max_w32, 4 * inst_w4(s));
    }
    max_rows = std::max(max_rows, rows);
    max_vecs = std::max(max_vecs, vecs);
    max_edges = std::max(max_edges, edges);
    max_n = std::max(max_n, w.second - w.first);
  }
  B.n_rows.reserve(max_n);
  B.n_cols.reserve(max_n);
  B.bad.reserve(1);
  B.w4.reserve(max_n);
  B.lshift.reserve(max_n);
  B.row_base.reserve(max_n);
  B.vec_base.reserve(max_n);
  B.delta.reserve(max_n);
  B.total.reserve(max_n);
  B.rounds.reserve(max_n);
  B.active.reserve(max_n);
  B.act.reserve(max_n);
  B.uprefix.reserve(max_n + 1);
  B.n_act.reserve(1);
  B.u_total.reserve(1);
  B.eoff.reserve(max_n + 1);
  B.deg.reserve(max_rows + 1);
  B.off.reserve(max_rows + 1);
  B.cursor.reserve(max_rows + 1);
  B.sums.reserve(ceil_div(max_rows + 1, SC_TILE) + 2);
  B.nbr.reserve(max_edges);
  B.f0.reserve(max_rows);
  B.f1.reserve(max_rows);
  B.F.reserve(max_vecs);
  B.D0.reserve(max_vecs);
  B.D1.reserve(max_vecs);
  B.bytes.reserve(1);
  DBuf<uint64_t> d_counts(ctx, max_n), d_fps(ctx, max_n), d_tpw(ctx, max_w32), d_tb(ctx, 1024);
  DBuf<uint32_t> d_src_w(ctx, 1), d_dst_w(ctx, 1);
  {
    std::vector<uint64_t> tpw, tb;
    poly_tables(max_w32, tpw, tb);
    SK_CUDA(cudaMemcpyAsync(d_tpw.p, tpw.data(), tpw.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(d_tb.p, tb.data(), 1024 * 8, cudaMemcpyHostToDevice, ctx->stream));
  }
  const bool profile = ctx->profiling;
  if (profile) SK_CUDA(cudaMemsetAsync(B.bytes.p, 0, 8, ctx->stream));
  BsView v = B.view(profile);
  v.status = ctx->d_status;
  const int grid = round_grid(ctx);
  const int R_graph = ctx->tune_bs_graph_rounds > 0 ? ctx->tune_bs_graph_rounds : 8;

  // The graph of R_graph rounds (even, so buffer parity is the same at every
  // replay) over the fixed buffers, captured once per call.
  cudaGraphExec_t exec = nullptr;
  uint32_t graph_n_inst = 0;
  auto capture = [&](uint32_t n_wave) {
    if (exec && graph_n_inst == n_wave) return;
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    cudaGraph_t g;
    SK_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    for (int r = 0; r < R_graph; r += 2) {
      k_bs_round<0><<<grid, BS_NT, 0, ctx->stream>>>(v);
      k_bs_book<<<1, BK_NT, 0, ctx->stream>>>(v, n_wave, 1);
      k_bs_round<1><<<grid, BS_NT, 0, ctx->stream>>>(v);
      k_bs_book<<<1, BK_NT, 0, ctx->stream>>>(v, n_wave, 1);
    }
    SK_CUDA(cudaStreamEndCapture(ctx->stream, &g));
    SK_CUDA(cudaGraphInstantiate(&exec, g, 0));
    cudaGraphDestroy(g);
    graph_n_inst = n_wave;
  };

  std::vector<uint32_t> h_rows, h_cols, h_w4;
  std::vector<uint8_t> h_ls, h_act;
  std::vector<uint64_t> h_rb, h_vb, h_eoff, h_up;
  std::vector<uint32_t> h_actl;
  for (auto& w : waves) {
    const uint32_t nw = w.second - w.first;
    h_rows.resize(nw);
    h_cols.resize(nw);
    h_w4.resize(nw);
    h_ls.resize(nw);
    h_rb.resize(nw);
    h_vb.resize(nw);
    h_eoff.resize(nw + 1);
    uint64_t rows = 0, vecs = 0, edges = 0;
    for (uint32_t k = 0; k < nw; k++) {
      const InstSpec& s = spec[order[w.first + k]];
      h_rows[k] = s.rows;
      h_cols[k] = s.cols;
      h_w4[k] = (uint32_t)inst_w4(s);
      h_ls[k] = (uint8_t)lanes_shift(h_w4[k]);
      h_rb[k] = rows;
      h_vb[k] = vecs;
      h_eoff[k] = edges;
      rows += s.rows;
      vecs += inst_vecs(s);
      edges += s.e1 - s.e0;
    }
    h_eoff[nw] = edges;
    // gather this wave's edges (contiguous per instance in the input)
    SK_CUDA(cudaMemcpyAsync(B.n_rows.p, h_rows.data(), nw * 4, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(B.n_cols.p, h_cols.data(), nw * 4, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(B.w4.p, h_w4.data(), nw * 4, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(B.lshift.p, h_ls.data(), nw, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(B.row_base.p, h_rb.data(), nw * 8, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(B.vec_base.p, h_vb.data(), nw * 8, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(B.eoff.p, h_eoff.data(), (nw + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    d_src_w.reserve(edges + 1);
    d_dst_w.reserve(edges + 1);
    for (uint32_t k = 0; k < nw; k++) {
      const InstSpec& s = spec[order[w.first + k]];
      if (s.e1 > s.e0) {
        SK_CUDA(cudaMemcpyAsync(d_src_w.p + h_eoff[k], d_src + s.e0, (s.e1 - s.e0) * 4, cudaMemcpyDeviceToDevice,
                                ctx->stream));
        SK_CUDA(cudaMemcpyAsync(d_dst_w.p + h_eoff[k], d_dst + s.e0, (s.e1 - s.e0) * 4, cudaMemcpyDeviceToDevice,
                                ctx->stream));
      }
    }
    SK_CUDA(cudaMemsetAsync(B.delta.p, 0, nw * 8, ctx->stream));
    SK_CUDA(cudaMemsetAsync(B.total.p, 0, nw * 8, ctx->stream));
    SK_CUDA(cudaMemsetAsync(B.rounds.p, 0, nw * 4, ctx->stream));
    SK_CUDA(cudaMemsetAsync(B.active.p, 1, nw, ctx->stream));
    SK_CUDA(cudaMemsetAsync(B.deg.p, 0, (rows + 1) * 4, ctx->stream));
    SK_CUDA(cudaMemsetAsync(B.F.p, 0, vecs * 16, ctx->stream));
    SK_CUDA(cudaMemsetAsync(d_counts.p, 0, nw * 8, ctx->stream));
    SK_CUDA(cudaMemsetAsync(d_fps.p, 0, nw * 8, ctx->stream));
    const unsigned eg = (unsigned)std::min<uint64_t>(ceil_div(std::max<uint64_t>(edges, 1), 256), ctx->num_sms * 16ull);
    if (edges) {
      SK_CUDA(cudaMemsetAsync(B.bad.p, 0, 4, ctx->stream));
      k_bs_degree<<<eg, 256, 0, ctx->stream>>>(d_src_w.p, d_dst_w.p, edges, B.eoff.p, nw, v, B.deg.p, B.bad.p);
      after_launch(ctx, "k_bs_degree");
      SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, B.bad.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
      SK_CUDA(cudaStreamSynchronize(ctx->stream));
      if ((uint32_t)ctx->h_scalar[0]) fail(STRATA_E_INVALID, "an edge endpoint lies outside its instance's nodes");
    }
    const uint64_t tiles = ceil_div(rows + 1, SC_TILE);
    k_bs_tile_sums<<<(unsigned)tiles, BS_NT, 0, ctx->stream>>>(B.deg.p, rows, B.sums.p);
    after_launch(ctx, "k_bs_tile_sums");
    scan_tile_sums(ctx, B.sums.p, tiles);
    k_bs_tile_write<<<(unsigned)tiles, BS_NT, 0, ctx->stream>>>(B.deg.p, rows, B.sums.p, B.off.p, B.cursor.p);
    after_launch(ctx, "k_bs_tile_write");
    if (edges) {
      k_bs_seed<<<eg, 256, 0, ctx->stream>>>(d_src_w.p, d_dst_w.p, edges, B.eoff.p, nw, v, B.cursor.p, B.nbr.p);
      after_launch(ctx, "k_bs_seed");
    }
    k_bs_flags0<<<(unsigned)std::min<uint64_t>(ceil_div(std::max<uint64_t>(rows, 1), 256), ctx->num_sms * 16ull), 256,
                  0, ctx->stream>>>(B.off.p, rows, B.f0.p);
    after_launch(ctx, "k_bs_flags0");
    SK_CUDA(cudaMemcpyAsync(B.D0.p, B.F.p, vecs * 16, cudaMemcpyDeviceToDevice, ctx->stream));
    k_bs_book<<<1, BK_NT, 0, ctx->stream>>>(v, nw, 0);
    after_launch(ctx, "k_bs_book");
    // rounds
    const int kh = kprof_begin(ctx, K_BS_ROUND);
    if (mode == 0) {
      capture(nw);
      while (true) {
        SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, B.n_act.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
        SK_CUDA(cudaStreamSynchronize(ctx->stream));
        if ((uint32_t)ctx->h_scalar[0] == 0) break;
        SK_CUDA(cudaGraphLaunch(exec, ctx->stream));
        R.graph_launches++;
        R.round_launches += R_graph;
        ctx->launches += 2 * (uint64_t)R_graph;
      }
    } else {
      int par = 0;
      while (true) {
        SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, B.n_act.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
        SK_CUDA(cudaStreamSynchronize(ctx->stream));
        if ((uint32_t)ctx->h_scalar[0] == 0) break;
        if (par == 0) k_bs_round<0><<<grid, BS_NT, 0, ctx->stream>>>(v);
        else k_bs_round<1><<<grid, BS_NT, 0, ctx->stream>>>(v);
        after_launch(ctx, "k_bs_round");
        k_bs_book<<<1, BK_NT, 0, ctx->stream>>>(v, nw, 1);
        after_launch(ctx, "k_bs_book");
        R.round_launches++;
        par ^= 1;
      }
    }
    kprof_end(ctx, kh, 0);
    // summaries: every instance of the wave as a unit range
    h_up.resize(nw + 1);
    h_actl.resize(nw);
    uint64_t acc = 0;
    for (uint32_t k = 0; k < nw; k++) {
      h_actl[k] = k;
      h_up[k] = acc;
      acc += ceil_div(h_rows[k], 32u >> h_ls[k]);
    }
    h_up[nw] = acc;
    const uint32_t nw32 = nw;
    SK_CUDA(cudaMemcpyAsync(B.act.p, h_actl.data(), nw * 4, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(B.uprefix.p, h_up.data(), (nw + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(B.n_act.p, &nw32, 4, cudaMemcpyHostToDevice, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(B.u_total.p, &acc, 8, cudaMemcpyHostToDevice, ctx->stream));
    if (want_fp) {
      k_bs_final<<<grid, BS_NT, 0, ctx->stream>>>(v, d_tpw.p, d_tb.p, d_counts.p, d_fps.p);
      after_launch(ctx, "k_bs_final");
    }
    std::vector<uint64_t> c(nw), f(nw), t(nw);
    std::vector<uint32_t> r(nw);
    SK_CUDA(cudaMemcpyAsync(c.data(), d_counts.p, nw * 8, cudaMemcpyDeviceToHost, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(f.data(), d_fps.p, nw * 8, cudaMemcpyDeviceToHost, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(t.data(), B.total.p, nw * 8, cudaMemcpyDeviceToHost, ctx->stream));
    SK_CUDA(cudaMemcpyAsync(r.data(), B.rounds.p, nw * 4, cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
    for (uint32_t k = 0; k < nw; k++) {
      const uint32_t i = order[w.first + k];
      R.counts[i] = want_fp ? c[k] : t[k];
      R.fps[i] = f[k];
      R.totals[i] = t[k];
      R.rounds[i] = r[k];
      R.rounds_max = std::max(R.rounds_max, r[k]);
      if (want_fp && c[k] != t[k]) fail(STRATA_E_CUDA, "bit-row popcount disagrees with the summed Δ sizes");
    }
    R.waves++;
  }
  if (profile) {
    uint64_t b = 0;
    read_u64(ctx, B.bytes.p, &b, 1);
    R.bytes = b;
    kprof_add_last(ctx, K_BS_ROUND, b);
  }
  if (exec) cudaGraphExecDestroy(exec);
}

// ---- one rank's share of a sharded closure ---------------------------------
// The rank owns path rows X ∈ [lo, lo + rows) (local row x = X - lo), each W4
// uint4 words over the Z domain.  A round reads Δ(Y) of every node from the
// gathered matrix Dfull (all ranks' slices of the previous round, rank r's
// slice = rows [r·per, r·per + per)) with its byte flags ffull, and writes
// Δ'(X) of its own rows into Dmine / fmine:
//     Δ'(X) = ( ∪_{Y ∈ out(X)} Δ(Y) ) ∖ path(X),   path(X) ∪= Δ'(X)
// the same round as k_bs_round, one warp per unit of 32 / L rows.
struct ShardView {
  uint32_t rows, n, W;
  int ls;                // log2(lanes per row)
  const uint64_t* off;   // rows + 1, local rows
  const uint32_t* nbr;   // global neighbour ids
  uint4* F;              // rows × W
  unsigned long long* delta;
  unsigned long long* bytes;  // algorithmic bytes (as k_bs_round counts them), or null
};

__global__ void __launch_bounds__(BS_NT) k_shard_round(ShardView v, const uint4* __restrict__ Dfull,
                                                       const uint8_t* __restrict__ ffull, uint4* __restrict__ Dmine,
                                                       uint8_t* __restrict__ fmine) {
  const int lane = threadIdx.x & 31;
  const int ls = v.ls;
  const uint32_t lpr = 1u << ls, sub = (uint32_t)lane >> ls, sl = (uint32_t)lane & (lpr - 1);
  const unsigned smask = ls == 5 ? 0xffffffffu : (((1u << lpr) - 1u) << (sub << ls));
  const uint32_t W = v.W;
  const uint64_t units = ((uint64_t)v.rows + (32u >> ls) - 1) / (32u >> ls);
  const uint64_t nwarps = (uint64_t)gridDim.x * (BS_NT / 32);
  uint64_t cnt = 0;
  unsigned long long moved = 0;
  for (uint64_t u = ((uint64_t)blockIdx.x * BS_NT + threadIdx.x) >> 5; u < units; u += nwarps) {
    const uint64_t x = u * (32u >> ls) + sub;
    const bool valid = x < v.rows;
    const uint64_t e0 = valid ? v.off[x] : 0, e1 = valid ? v.off[x + 1] : 0;
    bool any_y = false;
    for (uint64_t e = e0 + sl; e < e1; e += lpr) {
      const uint32_t y = v.nbr[e];
      if (y < v.n && ffull[y]) any_y = true;
    }
    const unsigned bal_y = __ballot_sync(kFull, any_y);  // every lane takes part
    const bool row_has = valid && (bal_y & smask) != 0u;
    bool row_any = false;
    if (valid) {
      uint32_t active_edges = 0, acc_words = 0;
      for (uint32_t c = sl; c < W; c += lpr) {
        uint4 nw = make_uint4(0u, 0u, 0u, 0u);
        if (row_has) {
          uint4 acc = make_uint4(0u, 0u, 0u, 0u);
          active_edges = 0;
          for (uint64_t e = e0; e < e1; e += 4) {
            uint32_t y[4];
            bool on[4];
#pragma unroll
            for (int q = 0; q < 4; q++) y[q] = e + q < e1 ? v.nbr[e + q] : 0xffffffffu;
#pragma unroll
            for (int q = 0; q < 4; q++) on[q] = y[q] < v.n && ffull[y[q]] != 0;
            uint4 d[4];
#pragma unroll
            for (int q = 0; q < 4; q++) d[q] = on[q] ? Dfull[(uint64_t)y[q] * W + c] : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
            for (int q = 0; q < 4; q++) {
              acc.x |= d[q].x;
              acc.y |= d[q].y;
              acc.z |= d[q].z;
              acc.w |= d[q].w;
              active_edges += on[q] ? 1u : 0u;
            }
          }
          if (any4(acc)) {
            acc_words++;
            uint4* fp = v.F + x * W + c;
            uint4 f = *fp;
            nw = make_uint4(acc.x & ~f.x, acc.y & ~f.y, acc.z & ~f.z, acc.w & ~f.w);
            if (any4(nw)) {
              *fp = make_uint4(f.x | nw.x, f.y | nw.y, f.z | nw.z, f.w | nw.w);
              cnt += popc4(nw);
              row_any = true;
            }
          }
        }
        Dmine[x * W + c] = nw;  // rows without Δ' are cleared too
      }
      if (v.bytes && row_has) {
        // this lane's words: Δ rows read, Δ' written, path read (and written
        // where bits are new); its share of the edge list and flags
        const uint64_t lw = (W > sl) ? (W - sl + lpr - 1) / lpr : 0;
        moved += lw * 16ull * (active_edges + 1) + acc_words * 32ull + (sl == 0 ? (e1 - e0) * 5ull : 0ull);
      }
    }
    const unsigned bal = __ballot_sync(kFull, row_any);
    if (valid && sl == 0) fmine[x] = (bal & smask) != 0u ? 1 : 0;
  }
  cnt = warp_sum(cnt);
  if (lane == 0 && cnt) atomicAdd(v.delta, (unsigned long long)cnt);
  if (v.bytes) {
    moved = warp_sum(moved);
    if (lane == 0 && moved) atomicAdd(v.bytes, moved);
  }
}

// Local out-degrees of the rank's rows; endpoints outside [0, n) set *bad.
__global__ void k_shard_degree(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, uint64_t m,
                               uint32_t n, uint32_t lo, uint32_t hi, uint64_t* deg, uint32_t* bad) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = src[e], b = dst[e];
    if (a >= n || b >= n) {
      atomicOr(bad, 1u);
      continue;
    }
    if (a >= lo && a < hi) atomicAdd(reinterpret_cast<unsigned long long*>(&deg[a - lo]), 1ull);
  }
}

// CSR fill (neighbour order within a row is free: the round ORs them) and
// the seed: path(X) = Δ0(X) = the out-neighbour bits of X.
__global__ void k_shard_fill(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, uint64_t m,
                             uint32_t n, uint32_t lo, uint32_t hi, uint32_t W, const uint64_t* __restrict__ off,
                             uint32_t* cursor, uint32_t* nbr, uint32_t* F, uint32_t* Dmine, uint8_t* fmine) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = src[e], b = dst[e];
    if (a >= n || b >= n || a < lo || a >= hi) continue;
    const uint32_t x = a - lo;
    nbr[off[x] + atomicAdd(&cursor[x], 1u)] = b;
    const uint64_t wd = (uint64_t)x * W * 4 + (b >> 5);
    atomicOr(&F[wd], 1u << (b & 31));
    atomicOr(&Dmine[wd], 1u << (b & 31));
    fmine[x] = 1;
  }
}

__global__ void k_shard_popc(const uint4* __restrict__ F, uint64_t words, unsigned long long* out) {
  uint64_t c = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (uint64_t)gridDim.x * blockDim.x)
    c += popc4(F[i]);
  c = warp_sum(c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, (unsigned long long)c);
}

// |path| and Σ mix64(X)·c^Z of the rank's rows (global X = lo + x); one warp
// per row.
__global__ void __launch_bounds__(BS_NT) k_shard_summary(const uint4* __restrict__ F, uint32_t rows, uint32_t W,
                                                         uint32_t lo, const uint64_t* __restrict__ tpw,
                                                         const uint64_t* __restrict__ tb_g, unsigned long long* out) {
  __shared__ uint64_t tb[4][256];
  for (int t = threadIdx.x; t < 1024; t += BS_NT) (&tb[0][0])[t] = tb_g[t];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = (uint64_t)gridDim.x * (BS_NT / 32);
  for (uint64_t x = ((uint64_t)blockIdx.x * BS_NT + threadIdx.x) >> 5; x < rows; x += nwarps) {
    uint64_t cnt = 0, poly = 0;
    for (uint32_t c = lane; c < W; c += 32) {
      const uint4 q = F[x * W + c];
      const uint32_t wd[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int h = 0; h < 4; h++) {
        const uint32_t w = wd[h];
        if (!w) continue;
        cnt += __popc(w);
        const uint64_t t = tb[0][w & 255] + tb[1][(w >> 8) & 255] + tb[2][(w >> 16) & 255] + tb[3][w >> 24];
        poly += tpw[4 * (uint64_t)c + h] * t;
      }
    }
    cnt = warp_sum(cnt);
    poly = warp_sum(poly);
    if (lane == 0) {
      uint64_t z = (uint64_t)lo + x + kPolyC;  // splitmix64 finalizer of the global X
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
      z ^= z >> 31;
      if (cnt) atomicAdd(&out[0], (unsigned long long)cnt);
      if (poly) atomicAdd(&out[1], (unsigned long long)(poly * z));
    }
  }
}

uint64_t bs_budget(strata_ctx* ctx) {
  uint64_t b = (uint64_t)((double)reusable_device_bytes(ctx) * 0.7);
  if (ctx->cap && ctx->cap > ctx->in_use) b = std::min<uint64_t>(b, ctx->cap - ctx->in_use);
  if (ctx->tune_bs_budget_mb > 0) b = std::min<uint64_t>(b, (uint64_t)ctx->tune_bs_budget_mb << 20);
  return b;
}

}  // namespace

// Batched driver (instances described on the host, edges on the device).
void tc_bool_batch(strata_ctx* ctx, uint32_t n_inst, const uint32_t* nodes, const uint64_t* edge_off,
                   const uint32_t* d_src, const uint32_t* d_dst, int mode, uint64_t* counts, uint64_t* fps,
                   uint32_t* rounds, strata_batch_stats* st) {
  if (st) std::memset(st, 0, sizeof(*st));
  reset_status(ctx);
  if (mode != 0 && mode != 1) fail(STRATA_E_INVALID, "mode must be 0 (batched) or 1 (one instance per launch)");
  std::vector<InstSpec> spec(n_inst);
  for (uint32_t i = 0; i < n_inst; i++) {
    if (edge_off[i + 1] < edge_off[i]) fail(STRATA_E_INVALID, "edge offsets must be non-decreasing");
    spec[i] = InstSpec{nodes[i], nodes[i], edge_off[i], edge_off[i + 1]};
  }
  const uint64_t l0 = ctx->launches;
  cudaEvent_t e0, e1;
  check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
  check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
  check_cuda(cudaEventRecord(e0, ctx->stream), "cudaEventRecord");
  release_all_cached(ctx);  // the waves are sized from what this context can reuse
  BsBuffers B(ctx);
  BsResult R;
  try {
    bs_run(ctx, spec, d_src, d_dst, mode, bs_budget(ctx), B, R, true);
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  check_cuda(cudaEventRecord(e1, ctx->stream), "cudaEventRecord");
  sync_and_check(ctx);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  kprof_collect(ctx);
  for (uint32_t i = 0; i < n_inst; i++) {
    if (counts) counts[i] = R.counts[i];
    if (fps) fps[i] = R.fps[i];
    if (rounds) rounds[i] = R.rounds[i];
  }
  if (st) {
    st->instances = n_inst;
    st->waves = R.waves;
    st->graph_launches = R.graph_launches;
    st->round_launches = R.round_launches;
    st->rounds_max = R.rounds_max;
    uint64_t tot = 0;
    for (auto c : R.counts) tot += c;
    st->result_tuples = tot;
    st->device_ms = ms;
    st->round_bytes = R.bytes;
    st->launches = ctx->launches - l0;
  }
}

// Single-instance Bool TC on bit rows: the relation comes back sorted by
// (X, Z) through the bitmap compaction.  Returns false when the bit matrices
// do not fit (the caller falls back to another plan).
bool tc_bool_bitset_fits(strata_ctx* ctx, uint64_t n_src, uint64_t n_dst, uint64_t m) {
  const InstSpec s{(uint32_t)n_src, (uint32_t)n_dst, 0, m};
  return n_src < (1ull << 32) && n_dst < (1ull << 32) && inst_bytes(s) <= std::min<uint64_t>(bs_budget(ctx), 8ull << 30);
}

template <class K>
uint64_t tc_bool_bitset(strata_ctx* ctx, const uint32_t* d_src, const uint32_t* d_dst, uint64_t m, uint64_t n_src,
                        uint64_t n_dst, int b1, DBuf<K>& out, uint64_t* rounds, uint64_t* round_bytes) {
  std::vector<InstSpec> spec{InstSpec{(uint32_t)n_src, (uint32_t)n_dst, 0, m}};
  BsBuffers B(ctx);
  BsResult R;
  bs_run(ctx, spec, d_src, d_dst, 0, UINT64_MAX, B, R, false);
  *rounds = R.rounds[0];
  *round_bytes = R.bytes;
  const uint64_t n = R.totals[0];
  const uint64_t w4 = inst_w4(spec[0]);
  const DenseLayout lay = dense_layout(b1, n_src, w4 * 128, false);
  out.reserve(n + 1);
  DBuf<uint64_t> states(ctx, dense_marks_states(lay.entries));
  const uint64_t got = dense_marks_compact<K, false, int32_t>(ctx, reinterpret_cast<uint32_t*>(B.F.p), lay, nullptr, out.p,
                                                     nullptr, n + 1, states.p);
  if (got != n) fail(STRATA_E_CUDA, "bit-row compaction count disagrees with the summed Δ sizes");
  return n;
}

// ---- sharded closure: one rank's share ------------------------------------
void tc_shard_init(strata_ctx* ctx, strata_tc_shard* sh, uint32_t n, const uint32_t* d_src, const uint32_t* d_dst,
                   uint64_t m, uint32_t rank, uint32_t world) {
  sh->n = n;
  sh->rank = rank;
  sh->world = world;
  sh->per = (uint32_t)ceil_div(n, world);
  sh->lo = std::min<uint64_t>((uint64_t)rank * sh->per, n);
  sh->hi = std::min<uint64_t>((uint64_t)sh->lo + sh->per, n);
  sh->w4 = (uint32_t)std::max<uint64_t>(1, ceil_div(n, 128));
  const uint32_t rows = sh->hi - sh->lo;
  sh->off.ctx = sh->nbr.ctx = sh->F.ctx = sh->acc.ctx = ctx;
  sh->acc.reserve(4);
  sh->off.reserve((uint64_t)rows + 2);
  SK_CUDA(cudaMemsetAsync(sh->off.p, 0, ((uint64_t)rows + 2) * 8, ctx->stream));
  SK_CUDA(cudaMemsetAsync(sh->acc.p, 0, 4 * 8, ctx->stream));
  const unsigned g = (unsigned)std::min<uint64_t>(ceil_div(m ? m : 1, BS_NT), (uint64_t)ctx->num_sms * 8);
  uint32_t* bad = reinterpret_cast<uint32_t*>(sh->acc.p + 3);
  k_shard_degree<<<g, BS_NT, 0, ctx->stream>>>(d_src, d_dst, m, n, sh->lo, sh->hi, sh->off.p, bad);
  after_launch(ctx, "k_shard_degree");
  scan_tile_sums(ctx, sh->off.p, rows);  // off[rows] = the rank's edges
  uint64_t edges, flag;
  read_u64(ctx, sh->off.p + rows, &edges, 1);
  read_u64(ctx, reinterpret_cast<const uint64_t*>(sh->acc.p + 3), &flag, 1);
  if ((uint32_t)flag) fail(STRATA_E_INVALID, "an edge endpoint is outside [0, n_nodes)");
  sh->n_edges = edges;
  sh->nbr.reserve(edges + 1);
  sh->F.reserve((uint64_t)sh->per * sh->w4 + 1);
  sh->src = d_src;
  sh->dst = d_dst;
  sh->m = m;
}

uint64_t tc_shard_seed(strata_ctx* ctx, strata_tc_shard* sh, uint4* Dmine, uint8_t* fmine) {
  const uint64_t vecs = (uint64_t)sh->per * sh->w4;
  SK_CUDA(cudaMemsetAsync(sh->F.p, 0, vecs * 16, ctx->stream));
  SK_CUDA(cudaMemsetAsync(Dmine, 0, vecs * 16, ctx->stream));
  SK_CUDA(cudaMemsetAsync(fmine, 0, sh->per, ctx->stream));
  DBuf<uint32_t> cursor(ctx, (uint64_t)(sh->hi - sh->lo) + 1);
  SK_CUDA(cudaMemsetAsync(cursor.p, 0, ((uint64_t)(sh->hi - sh->lo) + 1) * 4, ctx->stream));
  const unsigned g = (unsigned)std::min<uint64_t>(ceil_div(sh->m ? sh->m : 1, BS_NT), (uint64_t)ctx->num_sms * 8);
  k_shard_fill<<<g, BS_NT, 0, ctx->stream>>>(sh->src, sh->dst, sh->m, sh->n, sh->lo, sh->hi, sh->w4, sh->off.p,
                                             cursor.p, sh->nbr.p, reinterpret_cast<uint32_t*>(sh->F.p),
                                             reinterpret_cast<uint32_t*>(Dmine), fmine);
  after_launch(ctx, "k_shard_fill");
  SK_CUDA(cudaMemsetAsync(sh->acc.p, 0, 8, ctx->stream));
  k_shard_popc<<<(unsigned)std::min<uint64_t>(ceil_div(vecs ? vecs : 1, BS_NT), (uint64_t)ctx->num_sms * 8), BS_NT, 0,
                 ctx->stream>>>(sh->F.p, vecs, sh->acc.p);
  after_launch(ctx, "k_shard_popc");
  uint64_t c;
  read_u64(ctx, reinterpret_cast<const uint64_t*>(sh->acc.p), &c, 1);
  sync_and_check(ctx);
  // The rounds read only nbr / F: drop the caller's columns, which need not
  // outlive this call.
  sh->src = sh->dst = nullptr;
  sh->seeded = true;
  return c;  // |Δ0| of the rank's rows (distinct edges)
}

uint64_t tc_shard_round(strata_ctx* ctx, strata_tc_shard* sh, const uint4* Dfull, const uint8_t* ffull, uint4* Dmine,
                        uint8_t* fmine) {
  ShardView v{};
  v.rows = sh->hi - sh->lo;
  v.n = sh->n;
  v.W = sh->w4;
  v.ls = (int)lanes_shift(sh->w4);
  v.off = sh->off.p;
  v.nbr = sh->nbr.p;
  v.F = sh->F.p;
  v.delta = sh->acc.p;
  v.bytes = ctx->profiling ? sh->acc.p + 1 : nullptr;
  SK_CUDA(cudaMemsetAsync(sh->acc.p, 0, 16, ctx->stream));
  const uint64_t units = ceil_div((uint64_t)v.rows, 32u >> v.ls);
  int kh = -1;
  if (units) {
    const unsigned g = (unsigned)std::min<uint64_t>(ceil_div(units, BS_NT / 32), (uint64_t)ctx->num_sms * 8);
    kh = kprof_begin(ctx, K_SHARD_ROUND);
    k_shard_round<<<g, BS_NT, 0, ctx->stream>>>(v, Dfull, ffull, Dmine, fmine);
    kprof_end(ctx, kh, 0);
    after_launch(ctx, "k_shard_round");
  }
  uint64_t c[2];
  read_u64(ctx, reinterpret_cast<const uint64_t*>(sh->acc.p), c, 2);
  sync_and_check(ctx);
  if (kh >= 0) ctx->krecs[kh].bytes = c[1];
  return c[0];
}

void tc_shard_summary(strata_ctx* ctx, strata_tc_shard* sh, uint64_t* count, uint64_t* fp) {
  std::vector<uint64_t> tpw, tb;
  poly_tables((uint64_t)sh->w4 * 4, tpw, tb);
  DBuf<uint64_t> d_tpw(ctx, tpw.size()), d_tb(ctx, 1024);
  SK_CUDA(cudaMemcpyAsync(d_tpw.p, tpw.data(), tpw.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  SK_CUDA(cudaMemcpyAsync(d_tb.p, tb.data(), 1024 * 8, cudaMemcpyHostToDevice, ctx->stream));
  SK_CUDA(cudaMemsetAsync(sh->acc.p, 0, 16, ctx->stream));
  const uint32_t rows = sh->hi - sh->lo;
  if (rows) {
    const unsigned g = (unsigned)std::min<uint64_t>(ceil_div(rows, BS_NT / 32), (uint64_t)ctx->num_sms * 8);
    k_shard_summary<<<g, BS_NT, 0, ctx->stream>>>(sh->F.p, rows, sh->w4, sh->lo, d_tpw.p, d_tb.p, sh->acc.p);
    after_launch(ctx, "k_shard_summary");
  }
  uint64_t h[2];
  read_u64(ctx, reinterpret_cast<const uint64_t*>(sh->acc.p), h, 2);
  sync_and_check(ctx);
  *count = h[0];
  *fp = h[1];
}

// ---- sparse Δ exchange -------------------------------------------------------
// When a round's Δ' is sparse, the ranks exchange only its nonzero 128-bit
// words: each rank packs (global word index, low 64 bits, high 64 bits)
// triples of its slice, the triples of all ranks are gathered, and every rank
// rebuilds the full Δ and its row flags from them.  The bytes on the wire are
// 24 per nonzero word instead of the whole slice.

// Nonzero words of the slice, written at claimed slots below `cap`; *count
// receives the total (which may exceed cap).
__global__ void k_shard_pack(const uint4* __restrict__ D, uint64_t words, uint64_t row0_word, uint64_t cap,
                             long long* __restrict__ out, unsigned long long* count) {
  const int lane = threadIdx.x & 31;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < words; base += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t w = base + threadIdx.x;
    uint4 q = make_uint4(0u, 0u, 0u, 0u);
    if (w < words) q = D[w];
    const bool nz = any4(q);
    const unsigned bal = __ballot_sync(kFull, nz);
    if (!bal) continue;
    unsigned long long first = 0;
    if (lane == 0) first = atomicAdd(count, (unsigned long long)__popc(bal));
    first = __shfl_sync(kFull, first, 0);
    if (nz) {
      const uint64_t slot = first + __popc(bal & lanemask_lt());
      if (slot < cap) {
        out[3 * slot] = (long long)(row0_word + w);
        out[3 * slot + 1] = (long long)(((uint64_t)q.y << 32) | q.x);
        out[3 * slot + 2] = (long long)(((uint64_t)q.w << 32) | q.z);
      }
    }
  }
}

// Scatter gathered triples into the (cleared) full Δ; entries with index -1
// are padding, indexes past the matrix are skipped and flagged.
__global__ void k_shard_unpack(const long long* __restrict__ in, uint64_t n, uint4* __restrict__ D, uint64_t words,
                               uint32_t W, uint8_t* __restrict__ flags, uint32_t* status) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const long long idx = in[3 * i];
    if (idx < 0) continue;
    if ((uint64_t)idx >= words) {
      atomicOr(status, ST_BOUNDS);
      continue;
    }
    const uint64_t lo = (uint64_t)in[3 * i + 1], hi = (uint64_t)in[3 * i + 2];
    D[idx] = make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32));
    flags[(uint64_t)idx / W] = 1;
  }
}

uint64_t tc_shard_pack(strata_ctx* ctx, strata_tc_shard* sh, const uint4* Dmine, int64_t* out, uint64_t cap) {
  const uint64_t per = sh->per;
  const uint64_t words = per * sh->w4;
  DBuf<uint64_t> cnt(ctx, 1);
  SK_CUDA(cudaMemsetAsync(cnt.p, 0, 8, ctx->stream));
  if (cap) SK_CUDA(cudaMemsetAsync(out, 0xff, cap * 24, ctx->stream));  // padding: index -1
  if (words) {
    const unsigned g = (unsigned)std::min<uint64_t>(ceil_div(words, 256), (uint64_t)ctx->num_sms * 8);
    k_shard_pack<<<g, 256, 0, ctx->stream>>>(Dmine, words, (uint64_t)sh->rank * per * sh->w4, cap,
                                             reinterpret_cast<long long*>(out),
                                             reinterpret_cast<unsigned long long*>(cnt.p));
    after_launch(ctx, "k_shard_pack");
  }
  uint64_t c;
  read_u64(ctx, cnt.p, &c, 1);
  sync_and_check(ctx);
  return c;
}

void tc_shard_unpack(strata_ctx* ctx, strata_tc_shard* sh, const int64_t* in, uint64_t n, uint4* Dfull,
                     uint8_t* ffull) {
  const uint64_t rows = (uint64_t)sh->per * sh->world, words = rows * sh->w4;
  SK_CUDA(cudaMemsetAsync(Dfull, 0, words * 16, ctx->stream));
  SK_CUDA(cudaMemsetAsync(ffull, 0, rows, ctx->stream));
  if (n) {
    const unsigned g = (unsigned)std::min<uint64_t>(ceil_div(n, 256), (uint64_t)ctx->num_sms * 8);
    k_shard_unpack<<<g, 256, 0, ctx->stream>>>(reinterpret_cast<const long long*>(in), n, Dfull, words, sh->w4,
                                               ffull, ctx->d_status);
    after_launch(ctx, "k_shard_unpack");
  }
  sync_and_check(ctx);
}

template uint64_t tc_bool_bitset<uint32_t>(strata_ctx*, const uint32_t*, const uint32_t*, uint64_t, uint64_t,
                                           uint64_t, int, DBuf<uint32_t>&, uint64_t*, uint64_t*);
template uint64_t tc_bool_bitset<uint64_t>(strata_ctx*, const uint32_t*, const uint32_t*, uint64_t, uint64_t,
                                           uint64_t, int, DBuf<uint64_t>&, uint64_t*, uint64_t*);

}  // namespace sk
