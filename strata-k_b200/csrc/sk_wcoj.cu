// sk_wcoj.cu — worst-case-optimal counting joins on a device CSR.
//
// The count aggregate  n(count<X>) :- e(X,Y), e(Y,Z), e(X,Z)  counts the body
// bindings (strata-eval/src/naive.rs:300-391, fold_aggregate Count :391).
// With out(x) the sorted successors of x in the set e, the bindings are
//     Σ_{(X,Y) ∈ e} |out(X) ∩ out(Y)|,
// a leapfrog of two sorted lists per edge.  The reference runs one thread per
// edge with a serial merge over an id-oriented CSR built on the host
// (strata-gpu/src/wcoj.rs:27-43, 99-131).  Here the CSR is built on the device
// (radix sort + run reduction + offsets) and one warp owns a source vertex X:
// it stages out(X) in shared memory, expands the concatenation of out(Y) over
// Y ∈ out(X) with a warp scan so the 32 lanes stream the successor lists with
// coalesced loads, and probes each candidate Z in the staged list.
#include "sk_ops.cuh"
#include "sk_prims.cuh"
#include "sk_rel.cuh"

namespace sk {
namespace {

constexpr int TC_WARPS = 8;
constexpr int TC_NT = TC_WARPS * 32;
constexpr uint32_t TC_STAGE = 1024;  // successor entries staged per warp

__device__ __forceinline__ bool bsearch_u32(const uint32_t* a, uint32_t n, uint32_t x) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo < n && a[lo] == x;
}

__global__ void __launch_bounds__(TC_NT)
    k_tri_count(const uint32_t* __restrict__ off, const uint32_t* __restrict__ nbr, uint64_t n_nodes,
                uint32_t* counter, unsigned long long* total, uint32_t u_lo, uint32_t u_hi) {
  __shared__ uint32_t s_list[TC_WARPS][TC_STAGE];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long count = 0;
  while (true) {
    uint32_t u = 0;
    if (lane == 0) u = u_lo + atomicAdd(counter, 1u);
    u = __shfl_sync(kFull, u, 0);
    if (u >= u_hi || u >= n_nodes) break;
    const uint32_t a0 = off[u], du = off[u + 1] - a0;
    if (du == 0) continue;
    const bool staged = du <= TC_STAGE;
    if (staged) {
      for (uint32_t k = lane; k < du; k += 32) s_list[warp][k] = nbr[a0 + k];
    }
    __syncwarp();
    const uint32_t* A = staged ? s_list[warp] : nbr + a0;
    for (uint32_t c = 0; c < du; c += 32) {
      const uint32_t i = c + lane;
      const bool valid = i < du;
      const uint32_t v = valid ? A[i] : 0u;
      const uint64_t dv = (valid && v < n_nodes) ? (uint64_t)(off[v + 1] - off[v]) : 0ull;
      const uint32_t sv = (valid && v < n_nodes) ? off[v] : 0u;
      const uint64_t incl = warp_incl_sum(dv);
      const uint64_t D = __shfl_sync(kFull, incl, 31);
      for (uint64_t base = 0; base < D; base += 32) {
        const uint64_t j = base + lane;
        const bool ok = j < D;
        // owner lane t = number of lanes whose inclusive prefix is <= j
        int t = 0;
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
          const uint64_t val = __shfl_sync(kFull, incl, t + s - 1);
          if (val <= j) t += s;
        }
        const uint64_t ex_t = __shfl_sync(kFull, incl - dv, t & 31);
        const uint32_t sv_t = __shfl_sync(kFull, sv, t & 31);
        if (ok) {
          const uint32_t w = nbr[sv_t + (j - ex_t)];
          if (bsearch_u32(A, du, w)) count++;
        }
      }
    }
    __syncwarp();
  }
  count = warp_sum(count);
  if (lane == 0 && count) atomicAdd(total, count);
}

// Filtered probe (default).  Most candidates Z of a warp's expansion are not
// in out(X): the warp also sets one bit per out(X) entry in a small
// shared-memory bitmap (hash of Z, 16 bits per entry up to 8,192 bits, so a
// non-member passes with probability <= 1 - e^(-1/16) ~ 6 %, a member always),
// answers most candidates with one shared-memory load, and queues the ones
// that pass; whenever 32 are queued the whole warp binary-searches them
// together, so the searches run without idle lanes.  Exact: the bitmap has no
// false negatives and every queued candidate is searched once.
constexpr uint32_t TF_WORDS = 256;  // 8,192-bit filter per warp
constexpr uint32_t TF_MIN = 8;      // out-degree from which the filter pays for its setup

__device__ __forceinline__ uint32_t tf_hash(uint32_t z, int lg) { return (z * 0x85EBCA77u) >> (32 - lg); }

__global__ void __launch_bounds__(TC_NT)
    k_tri_count_filt(const uint32_t* __restrict__ off, const uint32_t* __restrict__ nbr, uint64_t n_nodes,
                     uint32_t* counter, unsigned long long* total, uint32_t u_lo, uint32_t u_hi) {
  __shared__ uint32_t s_list[TC_WARPS][TC_STAGE];
  __shared__ uint32_t s_filt[TC_WARPS][TF_WORDS];
  __shared__ uint32_t s_q[TC_WARPS][64];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = lanemask_lt();
  uint32_t* q = s_q[warp];
  uint32_t* F = s_filt[warp];
  unsigned long long count = 0;
  while (true) {
    uint32_t u = 0;
    if (lane == 0) u = u_lo + atomicAdd(counter, 1u);
    u = __shfl_sync(kFull, u, 0);
    if (u >= u_hi || u >= n_nodes) break;
    const uint32_t a0 = off[u], du = off[u + 1] - a0;
    if (du == 0) continue;
    const bool staged = du <= TC_STAGE;
    const bool filt = staged && du >= TF_MIN;
    // filter size: 16 bits per entry, 512 .. 8,192 bits
    int lg = 9;
    while (filt && lg < 13 && (1u << lg) < 16u * du) lg++;
    if (staged) {
      for (uint32_t k = lane; k < du; k += 32) s_list[warp][k] = nbr[a0 + k];
    }
    if (filt) {
      for (uint32_t k = lane; k < (1u << (lg - 5)); k += 32) F[k] = 0u;
      __syncwarp();
      for (uint32_t k = lane; k < du; k += 32) {
        const uint32_t h = tf_hash(s_list[warp][k], lg);
        atomicOr(&F[h >> 5], 1u << (h & 31));
      }
    }
    __syncwarp();
    const uint32_t* A = staged ? s_list[warp] : nbr + a0;
    uint32_t qn = 0;  // queued candidates (uniform)
    for (uint32_t c = 0; c < du; c += 32) {
      const uint32_t i = c + lane;
      const bool valid = i < du;
      const uint32_t v = valid ? A[i] : 0u;
      const uint32_t dv = (valid && v < n_nodes) ? off[v + 1] - off[v] : 0u;
      const uint32_t sv = (valid && v < n_nodes) ? off[v] : 0u;
      const uint32_t incl = warp_incl_sum(dv);
      const uint32_t ex = incl - dv;
      const uint32_t D = __shfl_sync(kFull, incl, 31);
      for (uint32_t base = 0; base < D; base += 32) {
        const uint32_t j = base + lane;
        const bool ok = j < D;
        // owner lane t = number of lanes whose inclusive prefix is <= j
        int t = 0;
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
          const uint32_t val = __shfl_sync(kFull, incl, t + s - 1);
          if (val <= j) t += s;
        }
        const uint32_t ex_t = __shfl_sync(kFull, ex, t);
        const uint32_t sv_t = __shfl_sync(kFull, sv, t);
        const uint32_t w = ok ? nbr[sv_t + (j - ex_t)] : 0u;
        if (!filt) {
          if (ok && bsearch_u32(A, du, w)) count++;
          continue;
        }
        const uint32_t h = tf_hash(w, lg);
        const bool pass = ok && ((F[h >> 5] >> (h & 31)) & 1u);
        const unsigned bal = __ballot_sync(kFull, pass);
        if (pass) q[qn + __popc(bal & lt)] = w;
        qn += __popc(bal);
        __syncwarp();
        if (qn >= 32) {
          if (bsearch_u32(A, du, q[lane])) count++;
          __syncwarp();
          if ((uint32_t)lane + 32 < qn) q[lane] = q[lane + 32];
          qn -= 32;
          __syncwarp();
        }
      }
    }
    if (qn > 0 && (uint32_t)lane < qn && bsearch_u32(A, du, q[lane])) count++;
    __syncwarp();
  }
  count = warp_sum(count);
  if (lane == 0 && count) atomicAdd(total, count);
}

// Hash-probe variant (STRATA_KNOB_TRI_PROBE = 1; measured slower than the
// binary search on R-MAT-22, which stays the default: the 8 KB table per warp
// cuts residency to 24 warps per SM and the probe loop diverges).  The warp
// builds an open-addressing set of out(X) in
// its shared-memory table (size the next power of two >= 2·d+(X), at most
// TH_TAB, so at least half the slots stay empty and every probe chain ends at
// an empty slot), then streams the successor lists of Y ∈ out(X) exactly as
// above and answers each membership test with ~1-2 table reads instead of a
// ~log2(d+(X))-step binary search.  A vertex whose out-list does not fit
// falls back to the binary search over its list in global memory.
constexpr uint32_t TH_TAB = 2048;
constexpr uint32_t kEmpty = 0xffffffffu;

__device__ __forceinline__ uint32_t tri_hash(uint32_t z, int lg) { return (z * 0x9E3779B1u) >> (32 - lg); }

__global__ void __launch_bounds__(TC_NT)
    k_tri_count_hash(const uint32_t* __restrict__ off, const uint32_t* __restrict__ nbr, uint64_t n_nodes,
                     uint32_t* counter, unsigned long long* total, uint32_t u_lo, uint32_t u_hi) {
  extern __shared__ __align__(16) uint32_t s_tab[];  // TC_WARPS * TH_TAB
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t* tab = s_tab + warp * TH_TAB;
  unsigned long long count = 0;
  while (true) {
    uint32_t u = 0;
    if (lane == 0) u = u_lo + atomicAdd(counter, 1u);
    u = __shfl_sync(kFull, u, 0);
    if (u >= u_hi || u >= n_nodes) break;
    const uint32_t a0 = off[u], du = off[u + 1] - a0;
    if (du == 0) continue;
    const bool hashed = du <= TH_TAB / 2;
    int lg = 5;
    while (hashed && (1u << lg) < 2 * du) lg++;
    const uint32_t tmask = (1u << lg) - 1;
    if (hashed) {
      for (uint32_t k = lane; k <= tmask; k += 32) tab[k] = kEmpty;
      __syncwarp();
      for (uint32_t k = lane; k < du; k += 32) {
        const uint32_t z = nbr[a0 + k];
        uint32_t slot = tri_hash(z, lg);
        // at most tmask+1 steps: the table is at most half full
        for (uint32_t step = 0; step <= tmask; step++) {
          const uint32_t prev = atomicCAS(&tab[slot], kEmpty, z);
          if (prev == kEmpty || prev == z) break;
          slot = (slot + 1) & tmask;
        }
      }
      __syncwarp();
    }
    for (uint32_t c = 0; c < du; c += 32) {
      const uint32_t i = c + lane;
      const bool valid = i < du;
      const uint32_t v = valid ? nbr[a0 + i] : 0u;
      const uint32_t dv = (valid && v < n_nodes) ? off[v + 1] - off[v] : 0u;
      const uint32_t sv = (valid && v < n_nodes) ? off[v] : 0u;
      const uint32_t incl = warp_incl_sum(dv);
      const uint32_t ex = incl - dv;
      const uint32_t D = __shfl_sync(kFull, incl, 31);
      for (uint32_t base = 0; base < D; base += 32) {
        const uint32_t j = base + lane;
        int t = 0;
#pragma unroll
        for (int st = 16; st > 0; st >>= 1) {
          const uint32_t val = __shfl_sync(kFull, incl, t + st - 1);
          if (val <= j) t += st;
        }
        const uint32_t ex_t = __shfl_sync(kFull, ex, t);
        const uint32_t sv_t = __shfl_sync(kFull, sv, t);
        if (j < D) {
          const uint32_t w = nbr[sv_t + (j - ex_t)];
          if (hashed) {
            uint32_t slot = tri_hash(w, lg);
            for (uint32_t step = 0; step <= tmask; step++) {
              const uint32_t x = tab[slot];
              if (x == w) { count++; break; }
              if (x == kEmpty) break;
              slot = (slot + 1) & tmask;
            }
          } else if (bsearch_u32(nbr + a0, du, w)) {
            count++;
          }
        }
      }
    }
    __syncwarp();
  }
  count = warp_sum(count);
  if (lane == 0 && count) atomicAdd(total, count);
}

// K4 on a degree-oriented DAG, one warp per lowest-rank vertex u.  A 4-clique
// a < b < c < d (rank order) is counted exactly once, at u = a, v = b, w = c,
// z = d: the warp stages out(u) in shared memory, and for each v ∈ out(u)
// builds the common-successor set C(u,v) = out(u) ∩ out(v) as a sorted list
// in shared memory (the lanes stream out(v) with coalesced loads, probe the
// staged out(u), and a ballot compacts the hits in order).  Then every
// w ∈ C(u,v) expands its out-list with the same warp-cooperative expansion
// as the triangle count (a warp scan over the 32 lanes' degrees, owner lane
// found by a shuffle search) and each entry z is probed in C(u,v).
//   count(u) = Σ_{v ∈ out(u)} Σ_{w ∈ C(u,v)} |out(w) ∩ C(u,v)|.
// A launch handles the vertices whose out-degree lies in (d_lo, d_hi]; `cap`
// (≥ d_hi, a multiple of 32) sizes the two per-warp lists in dynamic shared
// memory: one launch with a small cap and 8 warps per block for the bulk of
// the vertices, one with the largest out-degree as cap for the rest.
__global__ void k_k4_warp(const uint32_t* __restrict__ off, const uint32_t* __restrict__ nbr, uint64_t n_nodes,
                          uint32_t d_lo, uint32_t d_hi, uint32_t cap, uint32_t* counter,
                          unsigned long long* total) {
  extern __shared__ __align__(16) uint32_t s_k4[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t* A = s_k4 + (size_t)warp * 2 * cap;  // out(u), staged
  uint32_t* CL = A + cap;                       // C(u, v), sorted
  unsigned long long count = 0;
  while (true) {
    uint32_t u = 0;
    if (lane == 0) u = atomicAdd(counter, 1u);
    u = __shfl_sync(kFull, u, 0);
    if (u >= n_nodes) break;
    const uint32_t a0 = off[u], du = off[u + 1] - a0;
    if (du <= d_lo || du > d_hi || du < 3) continue;
    for (uint32_t k = lane; k < du; k += 32) A[k] = nbr[a0 + k];
    __syncwarp();
    for (uint32_t i = 0; i < du; i++) {  // v = A[i] (lists are in id order, not rank order)
      const uint32_t v = A[i];
      if (v >= n_nodes) continue;
      const uint32_t v0 = off[v], dv = off[v + 1] - v0;
      uint32_t nc = 0;
      for (uint32_t c = 0; c < dv; c += 32) {
        const bool valid = c + lane < dv;
        const uint32_t z = valid ? nbr[v0 + c + lane] : 0u;
        const bool hit = valid && bsearch_u32(A, du, z);
        const unsigned bal = __ballot_sync(kFull, hit);
        const uint32_t pos = nc + __popc(bal & lanemask_lt());
        if (hit && pos < cap) CL[pos] = z;  // distinct successors: nc <= du <= cap
        nc += __popc(bal);
      }
      __syncwarp();
      nc = min(nc, cap);
      if (nc < 2) continue;
      for (uint32_t c = 0; c < nc; c += 32) {
        const bool valid = c + lane < nc;
        const uint32_t w = valid ? CL[c + lane] : 0u;
        const bool inr = valid && w < n_nodes;
        const uint32_t sw = inr ? off[w] : 0u;
        const uint32_t dw = inr ? off[w + 1] - sw : 0u;
        const uint32_t incl = warp_incl_sum(dw);
        const uint32_t ex = incl - dw;
        const uint32_t D = __shfl_sync(kFull, incl, 31);
        for (uint32_t base = 0; base < D; base += 32) {
          const uint32_t j = base + lane;
          int t = 0;
#pragma unroll
          for (int st = 16; st > 0; st >>= 1) {
            const uint32_t val = __shfl_sync(kFull, incl, t + st - 1);
            if (val <= j) t += st;
          }
          const uint32_t ex_t = __shfl_sync(kFull, ex, t);
          const uint32_t sw_t = __shfl_sync(kFull, sw, t);
          if (j < D && bsearch_u32(CL, nc, nbr[sw_t + (j - ex_t)])) count++;
        }
      }
      __syncwarp();
    }
    __syncwarp();
  }
  count = warp_sum(count);
  if (lane == 0 && count) atomicAdd(total, count);
}

__global__ void k_max_outdeg(const uint32_t* __restrict__ off, uint64_t n_nodes, unsigned int* out) {
  unsigned int m = 0;
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n_nodes; u += (uint64_t)gridDim.x * blockDim.x)
    m = max(m, off[u + 1] - off[u]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(kFull, m, o));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// Canonical undirected edge key (min << b) | max; self-loops become the key
// (2^b-1, 2^b-1), which no real edge can take and which sorts last.
template <class K>
__global__ void k_canon(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, uint64_t n, int bits,
                        K* __restrict__ keys) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t x = a[i], y = b[i];
  const K lo = x < y ? x : y, hi = x < y ? y : x;
  const K sent = (K)((K(1) << bits) - 1);
  keys[i] = (x == y) ? (K)((sent << bits) | sent) : (K)((lo << bits) | hi);
}

template <class K>
__global__ void k_degree(const K* __restrict__ keys, uint64_t m, int bits, uint32_t* __restrict__ deg) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const K k = keys[i];
  const K mask = (K)((K(1) << bits) - 1);
  atomicAdd(&deg[(uint64_t)(k >> bits)], 1u);
  atomicAdd(&deg[(uint64_t)(k & mask)], 1u);
}

// Orient each undirected edge from lower to higher (degree, id) rank.
template <class K>
__global__ void k_orient(K* __restrict__ keys, uint64_t m, int bits, const uint32_t* __restrict__ deg) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const K k = keys[i];
  const K mask = (K)((K(1) << bits) - 1);
  const K x = k >> bits, y = k & mask;
  const uint32_t dx = deg[(uint64_t)x], dy = deg[(uint64_t)y];
  const bool x_first = dx < dy || (dx == dy && x < y);
  keys[i] = x_first ? (K)((x << bits) | y) : (K)((y << bits) | x);
}

__global__ void k_sum_sq_deg(const uint32_t* __restrict__ off, uint64_t n_nodes, unsigned long long* out) {
  unsigned long long acc = 0;
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n_nodes; u += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long d = off[u + 1] - off[u];
    acc += d * d;
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}

__global__ void k_max_u64(const uint64_t* __restrict__ a, uint64_t n, unsigned long long* out) {
  unsigned long long m = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    m = a[i] > m ? a[i] : m;
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(kFull, m, o);
    m = t > m ? t : m;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void k_intern_map(const uint64_t* __restrict__ keys, uint64_t n, const uint64_t* __restrict__ table,
                             uint64_t m, uint32_t* __restrict__ ids) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  ids[i] = (uint32_t)lower_bound_dev(table, 0, m, keys[i]);
}

inline unsigned blocks(uint64_t n, int nt = 256) { return (unsigned)ceil_div(n ? n : 1, nt); }

// Σ over oriented edges (u, v) of d+(u) + d+(v): the successor-list entries
// the triangle count streams (its algorithmic bytes; profiling only).
template <class K>
__global__ void k_tri_list_sum(const K* __restrict__ keys, uint64_t m, int bits, const uint32_t* __restrict__ off,
                               uint64_t n_nodes, unsigned long long* out) {
  unsigned long long s = 0;
  const K mask = (K)((K(1) << bits) - 1);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t u = (uint64_t)(keys[i] >> bits), v = (uint64_t)(keys[i] & mask);
    if (u < n_nodes) s += off[u + 1] - off[u];
    if (v < n_nodes) s += off[v + 1] - off[v];
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

// Sort + dedup packed keys in `keys` (n), result in out (returns count).
template <class K>
uint64_t sort_unique(strata_ctx* ctx, DBuf<K>& keys, uint64_t n, int bits, DBuf<K>& out) {
  DBuf<K> alt(ctx, n + 1);
  K* kp = keys.p;
  K* ka = alt.p;
  uint32_t* vp = nullptr;
  uint32_t* va = nullptr;
  radix_sort<K, uint32_t>(ctx, &kp, &ka, &vp, &va, false, n, bits, true);
  out.reserve(n + 1);
  DBuf<uint64_t> cnt(ctx, 1);
  reduce_runs<K, int32_t, false>(ctx, kp, nullptr, n, out.p, nullptr, cnt.p);
  uint64_t r;
  read_u64(ctx, cnt.p, &r, 1);
  return r;
}

// Count via the warp-per-vertex kernel over a CSR built from sorted unique keys.
template <class K>
uint64_t tri_from_sorted(strata_ctx* ctx, const K* keys, uint64_t m, int bits, uint64_t n_nodes, uint64_t u_lo = 0,
                         uint64_t u_hi = ~0ull) {
  if (u_hi > n_nodes) u_hi = n_nodes;
  if (u_lo >= u_hi) return 0;
  DBuf<uint32_t> off(ctx, n_nodes + 1), nbr(ctx, m + 1);
  build_csr<K>(ctx, keys, m, bits, n_nodes, off.p, nbr.p);
  DBuf<uint64_t> acc(ctx, 3);  // count, vertex counter, list-entry sum
  SK_CUDA(cudaMemsetAsync(acc.p, 0, 24, ctx->stream));
  const unsigned grid = (unsigned)std::min<uint64_t>(ceil_div(n_nodes, TC_WARPS), (uint64_t)ctx->num_sms * 8);
  const int kh = kprof_begin(ctx, K_TRI_COUNT);
  if (ctx->tune_tri_probe == 0 || ctx->tune_tri_probe == 3) {
    k_tri_count_filt<<<grid ? grid : 1, TC_NT, 0, ctx->stream>>>(off.p, nbr.p, n_nodes,
                                                                 reinterpret_cast<uint32_t*>(acc.p + 1),
                                                                 reinterpret_cast<unsigned long long*>(acc.p),
                                                                 (uint32_t)u_lo, (uint32_t)u_hi);
  } else if (ctx->tune_tri_probe == 2) {
    k_tri_count<<<grid ? grid : 1, TC_NT, 0, ctx->stream>>>(off.p, nbr.p, n_nodes,
                                                            reinterpret_cast<uint32_t*>(acc.p + 1),
                                                            reinterpret_cast<unsigned long long*>(acc.p),
                                                            (uint32_t)u_lo, (uint32_t)u_hi);
  } else {
    const size_t smem = (size_t)TC_WARPS * TH_TAB * sizeof(uint32_t);
    SK_CUDA(cudaFuncSetAttribute(k_tri_count_hash, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_tri_count_hash<<<grid ? grid : 1, TC_NT, smem, ctx->stream>>>(off.p, nbr.p, n_nodes,
                                                                     reinterpret_cast<uint32_t*>(acc.p + 1),
                                                                     reinterpret_cast<unsigned long long*>(acc.p),
                                                                     (uint32_t)u_lo, (uint32_t)u_hi);
  }
  // Algorithmic bytes: every out-list once per incident oriented edge plus the
  // edge list and offsets, 4 B·Σ(d+(u)+d+(v)) + 8 B·M + 4 B·(N+1); the sum is
  // counted on the device after the timed launch when profiling.
  kprof_end(ctx, kh, 8 * m + 4 * (n_nodes + 1));
  after_launch(ctx, "k_tri_count");
  if (ctx->profiling && m) {
    k_tri_list_sum<K><<<(unsigned)std::min<uint64_t>(blocks(m), (uint64_t)ctx->num_sms * 8), 256, 0, ctx->stream>>>(
        keys, m, bits, off.p, n_nodes, reinterpret_cast<unsigned long long*>(acc.p + 2));
    after_launch(ctx, "k_tri_list_sum");
  }
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, acc.p, 24, cudaMemcpyDeviceToHost, ctx->stream));
  sync_and_check(ctx);
  const uint64_t r = ctx->h_scalar[0];
  if (ctx->profiling) kprof_add_last(ctx, K_TRI_COUNT, 4 * ctx->h_scalar[2]);
  kprof_collect(ctx);
  return r;
}

template <class K>
uint64_t pattern_impl(strata_ctx* ctx, const uint32_t* x, const uint32_t* y, uint64_t n, int b,
                      uint64_t n_nodes, uint64_t u_lo = 0, uint64_t u_hi = ~0ull) {
  DBuf<K> keys(ctx, n + 1), uniq;
  uniq.ctx = ctx;
  pack_pairs<K, int32_t, false>(ctx, x, y, nullptr, nullptr, n, b, keys.p, nullptr);
  const uint64_t m = sort_unique<K>(ctx, keys, n, 2 * b, uniq);
  return tri_from_sorted<K>(ctx, uniq.p, m, b, n_nodes, u_lo, u_hi);
}

// Canonicalize, dedup, drop self-loops, orient by (degree, id).  Leaves the
// oriented sorted keys in `out` and returns their count.
template <class K>
uint64_t oriented_edges(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n, int bits,
                        uint64_t n_nodes, bool by_degree, DBuf<K>& out) {
  DBuf<K> keys(ctx, n + 1), uniq;
  uniq.ctx = ctx;
  k_canon<K><<<blocks(n), 256, 0, ctx->stream>>>(a, b, n, bits, keys.p);
  after_launch(ctx, "k_canon");
  uint64_t m = sort_unique<K>(ctx, keys, n, 2 * bits, uniq);
  if (m) {
    K last;
    SK_CUDA(cudaMemcpyAsync(&last, uniq.p + (m - 1), sizeof(K), cudaMemcpyDeviceToHost, ctx->stream));
    SK_CUDA(cudaStreamSynchronize(ctx->stream));
    const K sent = (K)((K(1) << bits) - 1);
    if (last == (K)((sent << bits) | sent)) m--;
  }
  if (!by_degree || m == 0) {
    out = std::move(uniq);
    return m;
  }
  DBuf<uint32_t> deg(ctx, n_nodes + 1);
  SK_CUDA(cudaMemsetAsync(deg.p, 0, (n_nodes + 1) * 4, ctx->stream));
  k_degree<K><<<blocks(m), 256, 0, ctx->stream>>>(uniq.p, m, bits, deg.p);
  after_launch(ctx, "k_degree");
  k_orient<K><<<blocks(m), 256, 0, ctx->stream>>>(uniq.p, m, bits, deg.p);
  after_launch(ctx, "k_orient");
  DBuf<K> alt(ctx, m + 1);
  K* kp = uniq.p;
  K* ka = alt.p;
  uint32_t* vp = nullptr;
  uint32_t* va = nullptr;
  radix_sort<K, uint32_t>(ctx, &kp, &ka, &vp, &va, false, m, 2 * bits, true);
  if (kp == uniq.p) out = std::move(uniq);
  else out = std::move(alt);
  return m;
}

template <class K>
uint64_t tri_undirected_impl(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n, int bits,
                             uint64_t n_nodes) {
  DBuf<K> ori;
  ori.ctx = ctx;
  const uint64_t m = oriented_edges<K>(ctx, a, b, n, bits, n_nodes, true, ori);
  if (m == 0) return 0;
  return tri_from_sorted<K>(ctx, ori.p, m, bits, n_nodes);
}

template <class K>
uint64_t k4_impl(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n, int bits, uint64_t n_nodes) {
  DBuf<K> ori;
  ori.ctx = ctx;
  const uint64_t m = oriented_edges<K>(ctx, a, b, n, bits, n_nodes, true, ori);
  if (m == 0) return 0;
  DBuf<uint32_t> off(ctx, n_nodes + 1), nbr(ctx, m + 1);
  build_csr<K>(ctx, ori.p, m, bits, n_nodes, off.p, nbr.p);
  DBuf<uint64_t> acc(ctx, 3);  // count, two vertex counters, largest out-degree
  SK_CUDA(cudaMemsetAsync(acc.p, 0, 24, ctx->stream));
  unsigned int* maxdeg = reinterpret_cast<unsigned int*>(acc.p + 2);
  k_max_outdeg<<<(unsigned)std::min<uint64_t>(blocks(n_nodes), (uint64_t)ctx->num_sms * 8), 256, 0, ctx->stream>>>(
      off.p, n_nodes, maxdeg);
  after_launch(ctx, "k_max_outdeg");
  uint64_t md;
  read_u64(ctx, acc.p + 2, &md, 1);
  md &= 0xffffffffull;
  // Shared memory of one warp: two lists of `cap` ids.
  constexpr uint32_t kSmallCap = 512;
  constexpr size_t kSmemLimit = 200 * 1024;
  const uint32_t big_cap = (uint32_t)ceil_div(std::max<uint64_t>(md, 1), 32) * 32;
  if ((size_t)big_cap * 8 > kSmemLimit)
    fail(STRATA_E_UNSUPPORTED, "4-clique count: an oriented out-degree above 25,600 does not fit shared memory");
  const uint64_t grid_cap = (uint64_t)ctx->num_sms * 8;
  auto launch = [&](uint32_t d_lo, uint32_t d_hi, uint32_t cap, int warps, uint32_t* counter) {
    const size_t smem = (size_t)warps * 2 * cap * 4;
    SK_CUDA(cudaFuncSetAttribute(k_k4_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(ceil_div(n_nodes, warps), grid_cap));
    k_k4_warp<<<grid, warps * 32, smem, ctx->stream>>>(off.p, nbr.p, n_nodes, d_lo, d_hi, cap, counter,
                                                       reinterpret_cast<unsigned long long*>(acc.p));
    after_launch(ctx, "k_k4_warp");
  };
  uint32_t* counters = reinterpret_cast<uint32_t*>(acc.p + 1);
  launch(0, kSmallCap, kSmallCap, 8, counters);
  if (md > kSmallCap) {
    const int warps = (int)std::max<size_t>(1, std::min<size_t>(8, kSmemLimit / ((size_t)big_cap * 8)));
    launch(kSmallCap, (uint32_t)md, big_cap, warps, counters + 1);
  }
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, acc.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
  sync_and_check(ctx);
  return ctx->h_scalar[0];
}

template <class K>
uint64_t bpi_impl(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n, int bits, uint64_t n_nodes) {
  DBuf<K> ori;
  ori.ctx = ctx;
  const uint64_t m = oriented_edges<K>(ctx, a, b, n, bits, n_nodes, false, ori);
  if (m == 0) return 0;
  DBuf<uint32_t> off(ctx, n_nodes + 1), nbr(ctx, m + 1);
  build_csr<K>(ctx, ori.p, m, bits, n_nodes, off.p, nbr.p);
  DBuf<uint64_t> acc(ctx, 1);
  SK_CUDA(cudaMemsetAsync(acc.p, 0, 8, ctx->stream));
  k_sum_sq_deg<<<blocks(n_nodes), 256, 0, ctx->stream>>>(off.p, n_nodes, reinterpret_cast<unsigned long long*>(acc.p));
  after_launch(ctx, "k_sum_sq_deg");
  uint64_t r;
  read_u64(ctx, acc.p, &r, 1);
  return r;
}

struct Ids {
  int bits;
  uint64_t n_nodes;
};

Ids id_space(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n) {
  const uint32_t m = std::max(max_u32(ctx, a, n), max_u32(ctx, b, n));
  return Ids{std::max(1, bits_for(m)), (uint64_t)m + 1};
}

}  // namespace

uint64_t count_triangle_pattern(strata_ctx* ctx, const uint32_t* x, const uint32_t* y, uint64_t n) {
  reset_status(ctx);
  if (n == 0) return 0;
  const Ids I = id_space(ctx, x, y, n);
  if (2 * I.bits <= 32) return pattern_impl<uint32_t>(ctx, x, y, n, I.bits, I.n_nodes);
  return pattern_impl<uint64_t>(ctx, x, y, n, I.bits, I.n_nodes);
}

uint64_t count_triangle_pattern_range(strata_ctx* ctx, const uint32_t* x, const uint32_t* y, uint64_t n,
                                      uint64_t u_lo, uint64_t u_hi) {
  reset_status(ctx);
  if (n == 0 || u_lo >= u_hi) return 0;
  const Ids I = id_space(ctx, x, y, n);
  if (2 * I.bits <= 32) return pattern_impl<uint32_t>(ctx, x, y, n, I.bits, I.n_nodes, u_lo, u_hi);
  return pattern_impl<uint64_t>(ctx, x, y, n, I.bits, I.n_nodes, u_lo, u_hi);
}

uint64_t count_triangles_undirected(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n) {
  reset_status(ctx);
  if (n == 0) return 0;
  const Ids I = id_space(ctx, a, b, n);
  if (2 * I.bits <= 32) return tri_undirected_impl<uint32_t>(ctx, a, b, n, I.bits, I.n_nodes);
  return tri_undirected_impl<uint64_t>(ctx, a, b, n, I.bits, I.n_nodes);
}

uint64_t count_4cliques_undirected(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n) {
  reset_status(ctx);
  if (n == 0) return 0;
  const Ids I = id_space(ctx, a, b, n);
  if (2 * I.bits <= 32) return k4_impl<uint32_t>(ctx, a, b, n, I.bits, I.n_nodes);
  return k4_impl<uint64_t>(ctx, a, b, n, I.bits, I.n_nodes);
}

uint64_t binary_plan_intermediate(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n) {
  reset_status(ctx);
  if (n == 0) return 0;
  const Ids I = id_space(ctx, a, b, n);
  if (2 * I.bits <= 32) return bpi_impl<uint32_t>(ctx, a, b, n, I.bits, I.n_nodes);
  return bpi_impl<uint64_t>(ctx, a, b, n, I.bits, I.n_nodes);
}

uint64_t intern_terms(strata_ctx* ctx, const uint64_t* keys, uint64_t n, uint32_t* ids) {
  reset_status(ctx);
  if (n == 0) return 0;
  DBuf<uint64_t> mx(ctx, 1);
  SK_CUDA(cudaMemsetAsync(mx.p, 0, 8, ctx->stream));
  k_max_u64<<<(unsigned)std::min<uint64_t>(ceil_div(n, 256), (uint64_t)ctx->num_sms * 8), 256, 0, ctx->stream>>>(
      keys, n, reinterpret_cast<unsigned long long*>(mx.p));
  after_launch(ctx, "k_max_u64");
  uint64_t maxk;
  read_u64(ctx, mx.p, &maxk, 1);
  DBuf<uint64_t> copy(ctx, n + 1), table;
  table.ctx = ctx;
  SK_CUDA(cudaMemcpyAsync(copy.p, keys, n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
  const uint64_t m = sort_unique<uint64_t>(ctx, copy, n, std::max(1, bits_for(maxk)), table);
  k_intern_map<<<blocks(n), 256, 0, ctx->stream>>>(keys, n, table.p, m, ids);
  after_launch(ctx, "k_intern_map");
  sync_and_check(ctx);
  return m;
}

}  // namespace sk
