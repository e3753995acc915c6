// sk_radix.cu — stable LSD radix sort of packed tuple keys (onesweep).
//
// Replaces the reference's 64 one-bit split passes with three host
// round-trips each (strata-gpu/src/sort.rs:337-365, scan_flags :282-315).
// Design for sm_100a:
//   * one upfront kernel computes the digit histograms of every pass from a
//     single read of the keys (warp-privatised shared-memory counters with
//     match-any aggregation);
//   * each 8-bit pass is ONE kernel: a tile of NT*ITEMS keys (and its
//     values) arrives in shared memory by one bulk asynchronous copy each,
//     is ranked with a warp-level multisplit (by default each lane ORs its
//     bit into its digit's shared-memory peer mask; 8 ballots per item and
//     the match instruction are knob choices), the tile's
//     per-digit counts are published for a decoupled look-back, keys are
//     staged in shared memory in digit order with their source slot and
//     written out in runs (coalesced per digit), values fetched through the
//     source slot — no per-key value state stays in registers;
//   * only the significant `bits` of the key are sorted (a 26-bit key takes 4
//     passes, not 64) and passes whose digit is constant are skipped.
#include "sk_ops.cuh"
#include "sk_prims.cuh"

#include <type_traits>
#include <vector>

namespace sk {
namespace {

constexpr int RADIX = 256;
constexpr int NT = 256;  // threads per block == RADIX (one digit per thread)
constexpr int NW = NT / 32;
// Look-back words: a 2-bit state (A = tile count ready, P = inclusive prefix
// ready) above the count.  32-bit words carry counts below 2^30 (sorts of at
// most 2^30 - 1 keys); 64-bit words take the larger sorts.
template <class LB> struct LbTag { using type = LB; };
template <class LB> struct LbBits {
  static constexpr int S = 8 * sizeof(LB) - 2;
  static constexpr LB A = LB(1) << S;
  static constexpr LB P = LB(2) << S;
  static constexpr LB M = (LB(1) << S) - 1;
};

template <class K> struct RCfg;
template <> struct RCfg<uint32_t> { static constexpr int ITEMS = 15; };
template <> struct RCfg<uint64_t> { static constexpr int ITEMS = 9; };

// Digit histograms of passes [p0, p0 + np), np <= 4.  Each warp loads HI
// keys per lane warp-striped (coalesced) and counts into its own shared
// counters; when all 32 lanes of a full row hold the same digit (long runs of
// equal high digits are the common case for packed keys) one add of 32
// replaces 32 atomics.
template <class K>
__global__ void __launch_bounds__(NT) k_radix_hist(const K* __restrict__ keys, uint64_t n, int p0,
                                                   int np, uint32_t* __restrict__ hist) {
  constexpr int HI = 8;
  __shared__ uint32_t sh[4][NW][RADIX];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < 4 * NW * RADIX; i += NT) (&sh[0][0][0])[i] = 0;
  __syncthreads();
  const uint64_t chunk = (uint64_t)NT * HI;
  for (uint64_t b0 = (uint64_t)blockIdx.x * chunk; b0 < n; b0 += (uint64_t)gridDim.x * chunk) {
    const uint64_t wb = b0 + (uint64_t)warp * 32 * HI;
    K k[HI];
#pragma unroll
    for (int j = 0; j < HI; j++) {
      const uint64_t i = wb + j * 32 + lane;
      k[j] = i < n ? keys[i] : K(0);
    }
    for (int p = 0; p < np; p++) {
      const int sh_bits = 8 * (p0 + p);
#pragma unroll
      for (int j = 0; j < HI; j++) {
        const uint64_t row = wb + j * 32;
        const uint32_t d = (uint32_t)(k[j] >> sh_bits) & 0xffu;
        if (row + 31 < n) {  // warp-uniform: the whole row is in range
          const uint32_t d0 = __shfl_sync(kFull, d, 0);
          if (__all_sync(kFull, d == d0)) {
            if (lane == 0) atomicAdd(&sh[p][warp][d0], 32u);
          } else {
            atomicAdd(&sh[p][warp][d], 1u);
          }
        } else if (row + lane < n) {
          atomicAdd(&sh[p][warp][d], 1u);
        }
      }
    }
  }
  __syncthreads();
  for (int i = tid; i < np * RADIX; i += NT) {
    const int p = i / RADIX, d = i % RADIX;
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < NW; w++) s += sh[p][w][d];
    if (s) atomicAdd(&hist[(p0 + p) * RADIX + d], s);
  }
}

// Exclusive scan of each pass's 256 bins (one block per pass).
__global__ void __launch_bounds__(NT) k_radix_bins(const uint32_t* __restrict__ hist,
                                                   uint32_t* __restrict__ binoff) {
  __shared__ uint32_t scratch[NW + 1];
  const uint32_t v = hist[blockIdx.x * RADIX + threadIdx.x];
  uint32_t tot;
  binoff[blockIdx.x * RADIX + threadIdx.x] = block_excl_sum<NT>(v, scratch, &tot);
}

// ---- bulk asynchronous copy of a tile into shared memory ---------------------
// One thread issues cp.async.bulk (global -> shared, completion counted in
// bytes on an mbarrier); the block waits on the barrier's phase with an
// iteration cap.  Addresses and sizes must be multiples of 16 bytes.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// true once phase `parity` of the barrier has completed; false after the cap
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < kSpinLimit; it++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

inline bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// Shared-memory layout of one pass: the tile's keys (loaded, then reused for
// the keys in digit order), its values in load order and, per sorted slot,
// the tile-local index the key came from.
// The source-slot region doubles as the per-warp peer masks of the
// shared-mask ranking, so it is at least NW * RADIX words.
template <class K, class V, bool HAS_V, int ITEMS>
constexpr size_t onesweep_smem() {
  constexpr size_t T = (size_t)NT * ITEMS;
  constexpr size_t src = HAS_V ? T * sizeof(uint16_t) : 0;
  constexpr size_t peer = (size_t)NW * RADIX * sizeof(uint32_t);
  return T * sizeof(K) + (HAS_V ? T * sizeof(V) : 0) + (src > peer ? src : peer);
}

// One stable 8-bit pass over tile `tile` (claimed in launch order).
//  1. thread 0 starts bulk copies of the tile's keys and values into shared
//     memory (full tiles with 16-byte aligned rows; otherwise plain loads);
//  2. every warp ranks its 32*ITEMS keys (warp-striped, so a warp's keys are
//     consecutive) with a warp multisplit against per-warp digit counters;
//  3. the tile's digit counts go out for the decoupled look-back and come
//     back as this tile's global base per digit;
//  4. keys are staged in digit order (with their source slot when values
//     ride along) and written out in runs, each value fetched from shared
//     memory through its source slot.
template <class K, class V, bool HAS_V, int ITEMS, int RANK, class LB = uint32_t>
__global__ void __launch_bounds__(NT, 4) k_onesweep(const K* __restrict__ kin, K* __restrict__ kout,
                                                 const V* __restrict__ vin, V* __restrict__ vout,
                                                 uint32_t n, int shift, int dbits,
                                                 const uint32_t* __restrict__ binoff,
                                                 LB* lookback, uint32_t* tile_counter,
                                                 uint32_t* status, int bulk_ok) {
  constexpr int rank_mode = RANK;  // 0 ballots, 1 match instruction, 2 shared masks
  constexpr uint32_t TILE = NT * ITEMS;
  static_assert(TILE <= 65536, "source slots are 16-bit");
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_whist[NW][RADIX];
  __shared__ uint32_t s_dstart[RADIX];
  __shared__ uint32_t s_goff[RADIX];
  __shared__ uint32_t s_scan[NW + 1];
  __shared__ __align__(8) uint64_t s_bar[2];
  extern __shared__ __align__(16) unsigned char s_raw[];
  K* s_keys = reinterpret_cast<K*>(s_raw);
  V* s_vin = reinterpret_cast<V*>(s_raw + (size_t)TILE * sizeof(K));
  uint16_t* s_src = reinterpret_cast<uint16_t*>(s_raw + (size_t)TILE * (sizeof(K) + (HAS_V ? sizeof(V) : 0)));
  uint32_t* s_peer = reinterpret_cast<uint32_t*>(s_src);  // [NW][RADIX], ranking only

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < NW * RADIX; i += NT) (&s_whist[0][0])[i] = 0;
  if (rank_mode == 2)
    for (int i = tid; i < NW * RADIX; i += NT) s_peer[i] = 0;
  if (tid == 0) {
    s_tile = atomicAdd(tile_counter, 1u);
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t base = tile * TILE;
  const uint32_t tile_n = min(TILE, n - base);
  const bool bulk = bulk_ok && tile_n == TILE;
  if (bulk) {
    if (tid == 0) {
      mbar_expect_tx(&s_bar[0], TILE * (uint32_t)sizeof(K));
      bulk_g2s(s_keys, kin + base, TILE * (uint32_t)sizeof(K), &s_bar[0]);
      if constexpr (HAS_V) {
        mbar_expect_tx(&s_bar[1], TILE * (uint32_t)sizeof(V));
        bulk_g2s(s_vin, vin + base, TILE * (uint32_t)sizeof(V), &s_bar[1]);
      }
    }
  } else {
    for (uint32_t i = tid; i < tile_n; i += NT) {
      s_keys[i] = kin[base + i];
      if constexpr (HAS_V) s_vin[i] = vin[base + i];
    }
  }
  const uint32_t dmask = (1u << dbits) - 1;
  const uint32_t wloc = (uint32_t)warp * 32u * ITEMS;  // this warp's first tile slot
  const unsigned lt = lanemask_lt();
  // every thread sees the keys (barrier phase, or the block barrier itself)
  const bool ok = __syncthreads_and(bulk ? mbar_wait(&s_bar[0], 0) : true);
  if (!ok) {
    // the copy never completed: record it, give the values' copy a bounded
    // wait too, and leave (successors' look-back waits are capped as well)
    if (tid == 0) atomicOr(status, ST_LOOKBACK_TIMEOUT);
    if (HAS_V) mbar_wait(&s_bar[1], 0);
    return;
  }

  K key[ITEMS];
  uint32_t rank[ITEMS];
#pragma unroll
  for (int j = 0; j < ITEMS; j++) {
    const uint32_t li = wloc + j * 32 + lane;
    key[j] = li < tile_n ? s_keys[li] : K(0);
  }
  // Warp-level multisplit: peers = lanes of this warp holding the same digit.
#pragma unroll
  for (int j = 0; j < ITEMS; j++) {
    const bool valid = wloc + j * 32 + lane < tile_n;
    const uint32_t d = (uint32_t)(key[j] >> shift) & dmask;
    unsigned peers;
    if (rank_mode == 2) {
      // shared-mask ranking: each lane ORs its bit into its digit's mask;
      // after the warp barrier the mask is the set of peers
      uint32_t* pm = &s_peer[warp * RADIX + d];
      if (valid) atomicOr(pm, 1u << lane);
      __syncwarp();
      peers = valid ? *pm : 0u;
    } else if (rank_mode == 1) {
      // one match instruction (invalid lanes carry a digit no valid lane has)
      peers = __match_any_sync(kFull, valid ? d : (0x100u | (uint32_t)lane));
    } else {
      peers = __ballot_sync(kFull, valid);
      if (dbits == 8) {
#pragma unroll
        for (int b = 0; b < 8; b++) {
          const unsigned bb = __ballot_sync(kFull, (d >> b) & 1u);
          peers &= ((d >> b) & 1u) ? bb : ~bb;
        }
      } else {
        for (int b = 0; b < dbits; b++) {
          const unsigned bb = __ballot_sync(kFull, (d >> b) & 1u);
          peers &= ((d >> b) & 1u) ? bb : ~bb;
        }
      }
    }
    const uint32_t prior = valid ? s_whist[warp][d] : 0u;
    rank[j] = prior + __popc(peers & lt);
    __syncwarp();
    if (valid && (peers & lt) == 0) {
      s_whist[warp][d] = prior + __popc(peers);
      if (rank_mode == 2) s_peer[warp * RADIX + d] = 0u;
    }
    __syncwarp();
  }
  __syncthreads();  // counters complete; every key of s_keys is in registers

  // Thread tid owns digit tid: warp-exclusive offsets and the tile count.
  uint32_t cnt = 0;
#pragma unroll
  for (int w = 0; w < NW; w++) {
    const uint32_t c = s_whist[w][tid];
    s_whist[w][tid] = cnt;
    cnt += c;
  }
  using LBB = LbBits<LB>;
  LB* lb = lookback + (size_t)tile * RADIX;
  st_volatile(&lb[tid], (tile == 0 ? LBB::P : LBB::A) | (LB)cnt);
  uint32_t tot;
  s_dstart[tid] = block_excl_sum<NT>(cnt, s_scan, &tot);

  LB excl = 0;  // keys of this digit in earlier tiles: below n < 2^32
  if (tile > 0) {
    bool timed_out = false;
    for (int64_t t = (int64_t)tile - 1; t >= 0; t--) {
      LB v;
      uint32_t it = 0;
      do {
        v = ld_volatile(&lookback[(size_t)t * RADIX + tid]);
      } while ((v >> LBB::S) == 0 && ++it < kSpinLimit);
      if ((v >> LBB::S) == 0) { timed_out = true; break; }
      excl += v & LBB::M;
      if ((v >> LBB::S) == 2) break;
    }
    if (timed_out) atomicOr(status, ST_LOOKBACK_TIMEOUT);
    st_volatile(&lb[tid], LBB::P | (excl + (LB)cnt));
  }
  s_goff[tid] = binoff[tid] + (uint32_t)excl - s_dstart[tid];
  __syncthreads();  // s_dstart, s_goff, warp offsets visible

  // Stage keys in digit order (and where each came from).
#pragma unroll
  for (int j = 0; j < ITEMS; j++) {
    const uint32_t li = wloc + j * 32 + lane;
    if (li < tile_n) {
      const uint32_t d = (uint32_t)(key[j] >> shift) & dmask;
      const uint32_t pos = s_dstart[d] + s_whist[warp][d] + rank[j];
      s_keys[pos] = key[j];
      if constexpr (HAS_V) s_src[pos] = (uint16_t)li;
    }
  }
  if constexpr (HAS_V) {
    if (bulk && !mbar_wait(&s_bar[1], 0) && tid == 0) atomicOr(status, ST_LOOKBACK_TIMEOUT);
  }
  __syncthreads();
#pragma unroll 4
  for (int j = 0; j < ITEMS; j++) {
    const uint32_t i = j * NT + tid;
    if (i < tile_n) {
      const K k = s_keys[i];
      const uint32_t d = (uint32_t)(k >> shift) & dmask;
      const uint32_t dst = s_goff[d] + i;
      if (dst < n) {
        kout[dst] = k;
        if constexpr (HAS_V) vout[dst] = s_vin[s_src[i]];
      } else {
        atomicOr(status, ST_BOUNDS);
      }
    }
  }
}

}  // namespace

namespace {

template <class K, class V, int ITEMS>
void radix_sort_impl(strata_ctx* ctx, K** keys, K** alt, V** vals, V** valt, bool has_vals,
                     uint64_t n, int bits, bool skip_trivial) {
  constexpr uint32_t TILE = NT * ITEMS;
  const int passes = (bits + 7) / 8;

  DBuf<uint32_t> hist(ctx, passes * RADIX + passes);
  uint32_t* counters = hist.p + passes * RADIX;
  SK_CUDA(cudaMemsetAsync(hist.p, 0, sizeof(uint32_t) * (passes * RADIX + passes), ctx->stream));
  const int hblocks = (int)std::min<uint64_t>(ceil_div(n, NT * 16), (uint64_t)ctx->num_sms * 4);
  for (int p0 = 0; p0 < passes; p0 += 4) {
    const int np = std::min(4, passes - p0);
    const int kh = kprof_begin(ctx, K_RADIX_HIST);
    k_radix_hist<K><<<hblocks, NT, 0, ctx->stream>>>(*keys, n, p0, np, hist.p);
    kprof_end(ctx, kh, n * sizeof(K));
    after_launch(ctx, "k_radix_hist");
  }
  DBuf<uint32_t> binoff(ctx, passes * RADIX);
  k_radix_bins<<<passes, NT, 0, ctx->stream>>>(hist.p, binoff.p);
  after_launch(ctx, "k_radix_bins");

  bool trivial[8] = {false, false, false, false, false, false, false, false};
  if (skip_trivial) {
    std::vector<uint32_t> h(passes * RADIX);
    SK_CUDA(cudaMemcpyAsync(h.data(), hist.p, sizeof(uint32_t) * passes * RADIX,
                            cudaMemcpyDeviceToHost, ctx->stream));
    SK_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int p = 0; p < passes; p++)
      for (int d = 0; d < RADIX; d++)
        if (h[p * RADIX + d] == n) trivial[p] = true;
  }

  const uint32_t ntiles = (uint32_t)ceil_div(n, TILE);
  // 64-bit look-back words once a digit's count can reach 2^30
  const bool wide_lb = n > kMaxSortN;
  const uint64_t lb_words = (uint64_t)ntiles * RADIX;
  const size_t lb_bytes = lb_words * (wide_lb ? 8 : 4);
  DBuf<uint64_t> lookback(ctx, (lb_bytes + 7) / 8);
  const size_t smem = has_vals ? onesweep_smem<K, V, true, ITEMS>() : onesweep_smem<K, V, false, ITEMS>();
  for (int p = 0; p < passes; p++) {
    if (trivial[p]) continue;
    SK_CUDA(cudaMemsetAsync(lookback.p, 0, lb_bytes, ctx->stream));
    const int dbits = std::min(8, bits - 8 * p);
    const int kh = kprof_begin(ctx, K_ONESWEEP);
    auto go = [&](auto rank_tag, auto lb_tag) {
      constexpr int RK = decltype(rank_tag)::value;
      using LB = typename decltype(lb_tag)::type;
      LB* lbp = reinterpret_cast<LB*>(lookback.p);
      if (has_vals) {
        auto kern = k_onesweep<K, V, true, ITEMS, RK, LB>;
        SK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<ntiles, NT, smem, ctx->stream>>>(*keys, *alt, *vals, *valt, (uint32_t)n, 8 * p, dbits,
                                                binoff.p + p * RADIX, lbp, counters + p, ctx->d_status,
                                                aligned16(*keys) && aligned16(*vals) ? 1 : 0);
      } else {
        auto kern = k_onesweep<K, V, false, ITEMS, RK, LB>;
        SK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<ntiles, NT, smem, ctx->stream>>>(*keys, *alt, nullptr, nullptr, (uint32_t)n, 8 * p, dbits,
                                                binoff.p + p * RADIX, lbp, counters + p, ctx->d_status,
                                                aligned16(*keys) ? 1 : 0);
      }
    };
    if (wide_lb)  // the large sorts take the default ranking
      go(std::integral_constant<int, 2>{}, LbTag<uint64_t>{});
    else
      switch (ctx->tune_sort_rank) {
        case 0: go(std::integral_constant<int, 0>{}, LbTag<uint32_t>{}); break;
        case 1: go(std::integral_constant<int, 1>{}, LbTag<uint32_t>{}); break;
        default: go(std::integral_constant<int, 2>{}, LbTag<uint32_t>{}); break;
      }
    kprof_end(ctx, kh, 2 * n * (sizeof(K) + (has_vals ? sizeof(V) : 0)));
    after_launch(ctx, "k_onesweep");
    std::swap(*keys, *alt);
    if (has_vals) std::swap(*vals, *valt);
  }
}

}  // namespace

// Keys per thread of the onesweep tile, selectable per context (the tuning
// knobs); the default is RCfg<K>::ITEMS.
int radix_items_choices(int key_bytes, int* out, int max_out) {
  static const int c4[] = {11, 15, 19, 23};
  static const int c8[] = {7, 9, 13};
  const int* c = key_bytes == 4 ? c4 : c8;
  const int nc = key_bytes == 4 ? 4 : 3;
  for (int i = 0; i < nc && i < max_out; i++) out[i] = c[i];
  return nc;
}

template <class K, class V>
void radix_sort(strata_ctx* ctx, K** keys, K** alt, V** vals, V** valt, bool has_vals,
                uint64_t n, int bits, bool skip_trivial) {
  if (n <= 1 || bits <= 0) return;
  if (n > kMaxSortKeys) fail(STRATA_E_UNSUPPORTED, "radix sort call limited to 2^32-1 keys");
  if (bits > (int)(8 * sizeof(K))) bits = 8 * sizeof(K);
  if constexpr (sizeof(K) == 4) {
    switch (ctx->tune_items4) {
      case 11: return radix_sort_impl<K, V, 11>(ctx, keys, alt, vals, valt, has_vals, n, bits, skip_trivial);
      case 19: return radix_sort_impl<K, V, 19>(ctx, keys, alt, vals, valt, has_vals, n, bits, skip_trivial);
      case 23: return radix_sort_impl<K, V, 23>(ctx, keys, alt, vals, valt, has_vals, n, bits, skip_trivial);
      default: return radix_sort_impl<K, V, 15>(ctx, keys, alt, vals, valt, has_vals, n, bits, skip_trivial);
    }
  } else {
    switch (ctx->tune_items8) {
      case 7: return radix_sort_impl<K, V, 7>(ctx, keys, alt, vals, valt, has_vals, n, bits, skip_trivial);
      case 13: return radix_sort_impl<K, V, 13>(ctx, keys, alt, vals, valt, has_vals, n, bits, skip_trivial);
      default: return radix_sort_impl<K, V, 9>(ctx, keys, alt, vals, valt, has_vals, n, bits, skip_trivial);
    }
  }
}

#define SK_INST_SORT(K, V)                                                                   \
  template void radix_sort<K, V>(strata_ctx*, K**, K**, V**, V**, bool, uint64_t, int, bool);
SK_INST_SORT(uint32_t, uint32_t)
SK_INST_SORT(uint32_t, uint64_t)
SK_INST_SORT(uint64_t, uint32_t)
SK_INST_SORT(uint64_t, uint64_t)
#undef SK_INST_SORT

// Variant for callers that cannot allocate: every temporary lives in the
// caller-supplied `scratch` (see sk_noalloc.cu).  Keys only, u32, the last
// pass always lands in `out`; no host synchronization inside.
uint64_t radix_sort_u32_static_bytes(uint64_t max_n) {
  constexpr uint32_t TILE = NT * RCfg<uint32_t>::ITEMS;
  const uint64_t tiles = ceil_div(max_n, TILE);
  // hist (4 passes) + bin offsets + tile counters + status + look-back + alt keys
  return 4 * RADIX * 4 + 4 * RADIX * 4 + 64 + 64 + tiles * RADIX * 4 + max_n * 4;
}

void radix_sort_u32_static(cudaStream_t stream, const uint32_t* in, uint32_t* out, uint64_t n, int bits,
                           unsigned char* scratch, uint64_t max_n, uint32_t* h_status) {
  constexpr int ITEMS = RCfg<uint32_t>::ITEMS;
  constexpr uint32_t TILE = NT * ITEMS;
  const int passes = (bits + 7) / 8;
  const uint32_t ntiles = (uint32_t)ceil_div(n, TILE);
  uint32_t* hist = reinterpret_cast<uint32_t*>(scratch);
  uint32_t* binoff = hist + 4 * RADIX;
  uint32_t* counters = binoff + 4 * RADIX;   // 16 slots
  uint32_t* status = counters + 16;          // 16 slots
  uint32_t* lookback = status + 16;
  uint32_t* alt = lookback + ceil_div(max_n, TILE) * RADIX;
  // Everything that must start at zero is cleared on every call.
  check_cuda(cudaMemsetAsync(hist, 0, (4 * RADIX + 4 * RADIX + 32) * 4, stream), "cudaMemsetAsync");
  const int hblocks = (int)std::min<uint64_t>(ceil_div(n, NT * 16), 148 * 4);
  k_radix_hist<uint32_t><<<hblocks, NT, 0, stream>>>(in, n, 0, passes, hist);
  k_radix_bins<<<passes, NT, 0, stream>>>(hist, binoff);
  const size_t smem = onesweep_smem<uint32_t, uint32_t, false, ITEMS>();
  const uint32_t* src = in;
  for (int p = 0; p < passes; p++) {
    // Ping-pong so that the last pass writes `out`.
    uint32_t* dst = ((passes - 1 - p) % 2 == 0) ? out : alt;
    check_cuda(cudaMemsetAsync(lookback, 0, sizeof(uint32_t) * ntiles * RADIX, stream), "cudaMemsetAsync");
    auto kern = k_onesweep<uint32_t, uint32_t, false, ITEMS, 2>;
    kern<<<ntiles, NT, smem, stream>>>(src, dst, nullptr, nullptr, (uint32_t)n, 8 * p, std::min(8, bits - 8 * p),
                                       binoff + p * RADIX, lookback, counters + p, status,
                                       aligned16(src) ? 1 : 0);
    src = dst;
  }
  check_cuda(cudaGetLastError(), "launch");
  check_cuda(cudaMemcpyAsync(h_status, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync");
}

}  // namespace sk
