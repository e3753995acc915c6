// sk_prims.cuh — device building blocks: warp/block scans and the bounded
// decoupled look-back used by every single-pass kernel (radix passes, offset
// scans, run reductions, merges).
//
// Look-back protocol: each tile publishes a word holding a 2-bit state (A =
// aggregate ready, P = inclusive prefix ready) and a count.  Tiles are claimed
// in launch order through an atomic counter, so every predecessor of a tile is
// resident or finished; waits are still capped at kSpinLimit iterations and a
// capped wait raises ST_LOOKBACK_TIMEOUT instead of spinning forever.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sk_common.cuh"

namespace sk {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <class T>
__device__ __forceinline__ T warp_incl_sum(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Block-wide exclusive sum for blockDim.x == NT (multiple of 32).  `scratch`
// needs NT/32 + 1 entries.  Returns the exclusive prefix; *total gets the sum.
template <int NT, class T>
__device__ __forceinline__ T block_excl_sum(T v, T* scratch, T* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T incl = warp_incl_sum(v);
  if (lane == 31) scratch[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    T w = (lane < NT / 32) ? scratch[lane] : T(0);
    T wi = warp_incl_sum(w);
    if (lane < NT / 32) scratch[lane] = wi - w;
    if (lane == NT / 32 - 1) scratch[NT / 32] = wi;
  }
  __syncthreads();
  T r = scratch[warp] + incl - v;
  *total = scratch[NT / 32];
  __syncthreads();
  return r;
}

// ---- 64-bit look-back (2 state bits on top, 62-bit value) -------------------
constexpr uint64_t kLbA = 1ull << 62;
constexpr uint64_t kLbP = 2ull << 62;
constexpr uint64_t kLbMask = (1ull << 62) - 1;

__device__ __forceinline__ uint64_t ld_volatile(const uint64_t* p) {
  return *reinterpret_cast<const volatile uint64_t*>(p);
}
__device__ __forceinline__ void st_volatile(uint64_t* p, uint64_t v) {
  *reinterpret_cast<volatile uint64_t*>(p) = v;
}
__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}
__device__ __forceinline__ void st_volatile(uint32_t* p, uint32_t v) {
  *reinterpret_cast<volatile uint32_t*>(p) = v;
}

// Executed by all 32 lanes of ONE warp.  Publishes `agg` for `tile`, walks the
// predecessors 32 at a time and returns the exclusive prefix (same on every
// lane).  `value` payloads are summed as 62-bit integers; `pack` lets callers
// carry two 31-bit counters in one word (sums never carry across because each
// half stays below 2^31).
__device__ __forceinline__ uint64_t warp_lookback(uint64_t* states, uint32_t tile, uint64_t agg,
                                                  uint32_t* status) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) st_volatile(&states[0], kLbP | agg);
    return 0;
  }
  if (lane == 0) st_volatile(&states[tile], kLbA | agg);
  uint64_t excl = 0;
  int64_t end = (int64_t)tile - 1;
  bool timed_out = false;
  while (true) {
    int64_t t = end - lane;
    uint64_t v = kLbP;  // virtual prefix 0 before tile 0
    if (t >= 0) {
      uint32_t it = 0;
      do {
        v = ld_volatile(&states[t]);
      } while ((v >> 62) == 0 && ++it < kSpinLimit);
      if ((v >> 62) == 0) { timed_out = true; v = kLbP; }
    }
    __syncwarp();
    unsigned pm = __ballot_sync(kFull, (v >> 62) == 2);
    int first_p = pm ? (__ffs(pm) - 1) : 32;
    uint64_t c = (lane <= first_p) ? (v & kLbMask) : 0;
    excl += warp_sum(c);
    if (pm) break;
    end -= 32;
  }
  if (__any_sync(kFull, timed_out) && lane == 0) atomicOr(status, ST_LOOKBACK_TIMEOUT);
  if (lane == 0) st_volatile(&states[tile], kLbP | (excl + agg));
  return excl;
}

// Dynamic tile id claimed in launch order (one atomic per block).
__device__ __forceinline__ uint32_t claim_tile(uint32_t* counter, uint32_t* smem_slot) {
  if (threadIdx.x == 0) *smem_slot = atomicAdd(counter, 1u);
  __syncthreads();
  return *smem_slot;
}

// ---- search helpers ------------------------------------------------------------
template <class K>
__device__ __forceinline__ uint64_t lower_bound_dev(const K* a, uint64_t lo, uint64_t hi, K x) {
  while (lo < hi) {
    uint64_t m = (lo + hi) >> 1;
    if (a[m] < x) lo = m + 1; else hi = m;
  }
  return lo;
}
template <class K>
__device__ __forceinline__ uint64_t upper_bound_dev(const K* a, uint64_t lo, uint64_t hi, K x) {
  while (lo < hi) {
    uint64_t m = (lo + hi) >> 1;
    if (a[m] <= x) lo = m + 1; else hi = m;
  }
  return lo;
}

// ---- Trop weights ----------------------------------------------------------------
// A device lane holds a weight CODE.  The reference's Weight is Finite(i64) |
// PosInf (strata-ir/src/trop.rs:35-40), so +inf must stay distinct from every
// finite value.  The two largest codes of a lane type are reserved:
//   WAbs = max      "absent" (the direct-addressed index's empty entry),
//   WInf = max - 1  +inf,
// and a finite value v is stored as the code v - s, at most max - 2.  The
// host picks the shift s per fixpoint from bounds on every sum the schedule
// can form (s in {0, 1, 2}: s > 0 only when those sums can reach i64::MAX,
// so a finite i64::MAX is representable) and checks that the smallest such
// sum still has a code.  Narrow (int32) lanes are only used with s = 0, when
// the host has proven every derived sum stays far inside the range, so they
// need no overflow test.
template <class W> struct WInf;
template <> struct WInf<int32_t> { static constexpr int32_t v = 0x7ffffffe; };
template <> struct WInf<int64_t> { static constexpr int64_t v = 0x7ffffffffffffffell; };
template <class W> struct WAbs;
template <> struct WAbs<int32_t> { static constexpr int32_t v = 0x7fffffff; };
template <> struct WAbs<int64_t> { static constexpr int64_t v = 0x7fffffffffffffffll; };
template <class W> struct WFinMax;  // largest finite code
template <> struct WFinMax<int32_t> { static constexpr int32_t v = 0x7ffffffd; };
template <> struct WFinMax<int64_t> { static constexpr int64_t v = 0x7ffffffffffffffdll; };

__device__ __forceinline__ int32_t trop_mul(int32_t a, int32_t b, int64_t s, uint32_t* flags) {
  (void)flags;
  (void)s;
  if (a == WInf<int32_t>::v || b == WInf<int32_t>::v) return WInf<int32_t>::v;
  return a + b;
}
// Checked i64 add with +inf absorption (strata-ir/src/trop.rs:52-62) on codes:
// values a + s and b + s, so the code of their sum is a + b + s.  A sum above
// i64::MAX (a code above WFinMax) or below i64::MIN is the reference's
// overflow error.
__device__ __forceinline__ int64_t trop_mul(int64_t a, int64_t b, int64_t s, uint32_t* flags) {
  if (a == WInf<int64_t>::v || b == WInf<int64_t>::v) return WInf<int64_t>::v;
  const long long as = a + s;  // a <= WFinMax and s <= 2: no wrap
  const long long r = (long long)((unsigned long long)as + (unsigned long long)b);
  if ((((as ^ r) & (b ^ r)) < 0) || r > WFinMax<int64_t>::v) {  // wrapped, or past i64::MAX
    *flags |= ST_OVERFLOW;
    return WInf<int64_t>::v;
  }
  return r;
}

}  // namespace sk
