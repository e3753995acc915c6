// sk_common.cuh — context, device memory, error and status plumbing shared by
// every translation unit of the engine.
//
// Errors inside the library are C++ exceptions (SkError) carrying a
// strata_status; every extern "C" entry point catches them and returns the
// code, storing the message in the context.  Device-side conditions (Trop
// overflow, a sentinel collision, a look-back wait that gave up) are bits in a
// per-context status word that kernels OR into and the host reads at each
// round boundary.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "../../include/strata_b200.h"

namespace sk {

// ---- device status bits -----------------------------------------------------
enum : uint32_t {
  ST_OVERFLOW = 1u,          // finite Trop (x) overflowed int64
  ST_SENTINEL = 2u,          // a finite input weight has no code in the fixpoint's weight lanes
  ST_LOOKBACK_TIMEOUT = 4u,  // decoupled look-back wait hit its iteration cap
  ST_BOUNDS = 8u,            // an index failed a bounds check and was skipped
  ST_PROOF_LEN = 16u,        // a provenance proof exceeded its literal capacity
};

// Iteration cap of every spin-wait in device code.  A wait that reaches it
// records ST_LOOKBACK_TIMEOUT and proceeds; the host turns that into
// STRATA_E_TIMEOUT.  Tiles are claimed in launch order, so a predecessor is
// always resident or finished and the cap is never reached in a correct run.
constexpr uint32_t kSpinLimit = 1u << 24;

struct SkError {
  strata_status code;
  std::string msg;
};

[[noreturn]] inline void fail(strata_status code, const std::string& msg) {
  throw SkError{code, msg};
}

inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    fail(e == cudaErrorMemoryAllocation ? STRATA_E_OOM : STRATA_E_CUDA,
         std::string(what) + ": " + cudaGetErrorString(e));
  }
}

#define SK_CUDA(call) ::sk::check_cuda((call), #call)

struct PhaseTimer;

}  // namespace sk

// The context: one device, one stream, a capped byte budget, a status word.
struct strata_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  uint64_t cap = 0;
  uint64_t in_use = 0;   // bytes of live blocks
  uint64_t cached = 0;   // bytes of freed blocks kept for reuse
  uint64_t peak = 0;
  std::unordered_map<void*, uint64_t> sizes;
  std::multimap<uint64_t, void*> free_blocks;  // size -> block, reused in stream order
  std::string last_error;
  uint32_t* d_status = nullptr;     // device status word
  uint32_t* h_status = nullptr;     // pinned mirror
  uint64_t* h_scalar = nullptr;     // pinned scratch for small D2H reads (8 slots)
  int num_sms = 148;
  cudaMemPool_t pool = nullptr;     // this context's pool (kept mapped between calls)
  int plan = 0;                     // 0 auto, 1 sort-merge, 2 direct-addressed
  int tune_items4 = 0;              // radix keys per thread, u32 keys (0 = default)
  int tune_items8 = 0;              // radix keys per thread, u64 keys (0 = default)
  int tune_sort_rank = 2;           // radix ranking: 0 bit ballots, 1 match instruction, 2 shared masks
  int tune_tri_probe = 0;           // triangle membership test: 1 hash set, 2 binary search, 0/3 bitmap filter
  int tune_bs_graph_rounds = 0;     // bit-row rounds per CUDA-graph replay (0 = 8)
  int tune_bs_blocks = 0;           // resident round-kernel blocks per SM (0 = occupancy limit)
  uint64_t tune_bs_budget_mb = 0;   // cap on a batch wave's device bytes, MiB (0 = 70% of free)
  int tune_dense_members = 0;       // members from which a Δ word takes the bit-lane expand (0 = 24)
  int64_t wshift = 0;               // weight code shift of the running fixpoint (value = code + wshift)
  bool force_wide = false;          // Trop fixpoints always in int64 lanes (STRATA_KNOB_WEIGHT_LANES = 8)
  bool profiling = false;
  uint64_t launches = 0;
  // Per-kernel CUDA-event accounting (enabled with profiling).
  struct KRec { int kid; cudaEvent_t a, b; uint64_t bytes; };
  std::vector<KRec> krecs;
  std::vector<cudaEvent_t> event_pool;
  struct KAgg { uint64_t launches = 0; double ms = 0; uint64_t bytes = 0; };
  KAgg kagg[16];
};

namespace sk {

// ---- allocation -------------------------------------------------------------

// Size classes: 256 B granules below 1 MiB, then steps of 1/8 of the power of
// two, so a block freed by one call fits the same request of the next call.
inline uint64_t size_class(uint64_t bytes) {
  if (bytes <= (1ull << 20)) return (bytes + 255) & ~uint64_t(255);
  int hb = 63 - __builtin_clzll(bytes);
  const uint64_t step = 1ull << (hb - 3);
  return (bytes + step - 1) & ~(step - 1);
}

inline void release_cached(strata_ctx* ctx, uint64_t need) {
  // Return cached blocks to the pool until `need` bytes fit under the cap.
  while (!ctx->free_blocks.empty() && ctx->cap && ctx->in_use + ctx->cached + need > ctx->cap) {
    auto it = std::prev(ctx->free_blocks.end());
    cudaFreeAsync(it->second, ctx->stream);
    ctx->cached -= it->first;
    ctx->free_blocks.erase(it);
  }
}

// Device bytes this context could obtain now: the device's free memory,
// plus what its pool holds unused, plus the blocks it keeps cached.
inline uint64_t reusable_device_bytes(strata_ctx* ctx) {
  size_t fr = 0, tot = 0;
  check_cuda(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo");
  uint64_t extra = ctx->cached;
  if (ctx->pool) {
    unsigned long long reserved = 0, used = 0;  // the attribute value type (cuuint64_t)
    if (cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
        cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
      extra += reserved - used;
  }
  return (uint64_t)fr + extra;
}

// Give every cached block back to the pool (before sizing large buffers).
inline void release_all_cached(strata_ctx* ctx) {
  for (auto& kv : ctx->free_blocks) cudaFreeAsync(kv.second, ctx->stream);
  ctx->free_blocks.clear();
  ctx->cached = 0;
}

inline void* dev_alloc(strata_ctx* ctx, uint64_t bytes) {
  if (bytes == 0) bytes = 16;
  bytes = size_class(bytes);
  // Reuse the smallest cached block that fits (all work is stream ordered on
  // ctx->stream, so a block freed earlier on it is free for later work).
  auto it = ctx->free_blocks.lower_bound(bytes);
  if (it != ctx->free_blocks.end() && it->first <= bytes + bytes / 4) {
    void* p = it->second;
    const uint64_t sz = it->first;
    ctx->free_blocks.erase(it);
    ctx->cached -= sz;
    ctx->sizes[p] = sz;
    ctx->in_use += sz;
    if (ctx->in_use > ctx->peak) ctx->peak = ctx->in_use;
    return p;
  }
  release_cached(ctx, bytes);
  if (ctx->cap && ctx->in_use + ctx->cached + bytes > ctx->cap) {
    fail(STRATA_E_OOM, "device memory cap reached: need " + std::to_string(bytes) +
                           " B with " + std::to_string(ctx->in_use) + " of " +
                           std::to_string(ctx->cap) + " B held");
  }
  void* p = nullptr;
  cudaError_t e = ctx->pool ? cudaMallocFromPoolAsync(&p, bytes, ctx->pool, ctx->stream)
                            : cudaMallocAsync(&p, bytes, ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    // Give the cached blocks back and try once more before failing.
    const uint64_t keep_cap = ctx->cap;
    ctx->cap = 1;
    release_cached(ctx, 0);
    ctx->cap = keep_cap;
    e = ctx->pool ? cudaMallocFromPoolAsync(&p, bytes, ctx->pool, ctx->stream)
                  : cudaMallocAsync(&p, bytes, ctx->stream);
    if (e != cudaSuccess && ctx->pool) {
      // The pool's free memory may be fragmented: return it to the device.
      cudaGetLastError();
      cudaStreamSynchronize(ctx->stream);
      cudaMemPoolTrimTo(ctx->pool, 0);
      e = cudaMallocFromPoolAsync(&p, bytes, ctx->pool, ctx->stream);
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      fail(STRATA_E_OOM, std::string("cudaMallocAsync(") + std::to_string(bytes) +
                             "): " + cudaGetErrorString(e));
    }
  }
  ctx->sizes[p] = bytes;
  ctx->in_use += bytes;
  if (ctx->in_use > ctx->peak) ctx->peak = ctx->in_use;
  return p;
}

inline void dev_free(strata_ctx* ctx, void* p) {
  if (!p) return;
  auto it = ctx->sizes.find(p);
  if (it == ctx->sizes.end()) {
    cudaFreeAsync(p, ctx->stream);
    return;
  }
  ctx->in_use -= it->second;
  ctx->cached += it->second;
  ctx->free_blocks.emplace(it->second, p);
  ctx->sizes.erase(it);
}

// Owning device buffer (RAII, stream-ordered free).
template <class T>
struct DBuf {
  strata_ctx* ctx = nullptr;
  T* p = nullptr;
  uint64_t cap = 0;  // elements
  DBuf() = default;
  DBuf(strata_ctx* c, uint64_t n) : ctx(c) { reserve(n); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : ctx(o.ctx), p(o.p), cap(o.cap) { o.p = nullptr; o.cap = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) {
      release();
      ctx = o.ctx; p = o.p; cap = o.cap;
      o.p = nullptr; o.cap = 0;
    }
    return *this;
  }
  ~DBuf() { release(); }
  void release() {
    if (p && ctx) dev_free(ctx, p);
    p = nullptr;
    cap = 0;
  }
  // Ensure capacity for n elements (contents not preserved when it grows).
  void reserve(uint64_t n) {
    if (n <= cap && p) return;
    release();
    uint64_t want = n < 64 ? 64 : n;
    p = static_cast<T*>(dev_alloc(ctx, want * sizeof(T)));
    cap = want;
  }
  // Grow geometrically (for per-round buffers that are reused).
  void reserve_grow(uint64_t n) {
    if (n <= cap && p) return;
    uint64_t want = cap ? cap : 64;
    while (want < n) want += want / 2 + 64;
    reserve(want);
  }
  // Give up ownership (the caller frees with dev_free).
  T* detach() {
    T* r = p;
    p = nullptr;
    cap = 0;
    return r;
  }
  void swap(DBuf& o) {
    std::swap(ctx, o.ctx);
    std::swap(p, o.p);
    std::swap(cap, o.cap);
  }
};

// ---- status word ------------------------------------------------------------

inline void reset_status(strata_ctx* ctx) {
  SK_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), ctx->stream));
}

// Synchronize and read the status word; throws on any device-side condition.
inline void sync_and_check(strata_ctx* ctx) {
  SK_CUDA(cudaMemcpyAsync(ctx->h_status, ctx->d_status, sizeof(uint32_t),
                          cudaMemcpyDeviceToHost, ctx->stream));
  SK_CUDA(cudaStreamSynchronize(ctx->stream));
  SK_CUDA(cudaGetLastError());
  uint32_t s = *ctx->h_status;
  if (s & ST_LOOKBACK_TIMEOUT) fail(STRATA_E_TIMEOUT, "a device look-back wait reached its cap");
  if (s & ST_BOUNDS) fail(STRATA_E_CUDA, "a device bounds check failed (index skipped)");
  if (s & ST_PROOF_LEN) fail(STRATA_E_UNSUPPORTED, "a provenance proof exceeded 32 literals");
  if (s & ST_OVERFLOW) fail(STRATA_E_OVERFLOW, "tropical weight overflow: a finite sum exceeds i64");
  if (s & ST_SENTINEL)
    fail(STRATA_E_WEIGHT_RANGE,
         "finite tropical weights span nearly all of i64 (sums within the round cap can reach both "
         "i64::MIN and i64::MAX): no 64-bit code keeps them apart from +inf");
}

// Read `count` u64 values from device memory (synchronizing).
inline void read_u64(strata_ctx* ctx, const uint64_t* d, uint64_t* out, int count) {
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, d, sizeof(uint64_t) * count,
                          cudaMemcpyDeviceToHost, ctx->stream));
  SK_CUDA(cudaStreamSynchronize(ctx->stream));
  std::memcpy(out, ctx->h_scalar, sizeof(uint64_t) * count);
}

inline void after_launch(strata_ctx* ctx, const char* name) {
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) fail(STRATA_E_CUDA, std::string("launch ") + name + ": " + cudaGetErrorString(e));
}

inline uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

inline int bits_for(uint64_t max_value) {  // bits needed to hold 0..max_value
  int b = 0;
  while (b < 64 && (max_value >> b) != 0) b++;
  return b;
}

// ---- per-kernel timing ----------------------------------------------------------
// Kernel ids reported by strata_ctx_kernel_stats.
enum KernelId : int {
  K_ONESWEEP = 0,
  K_EXPAND_EMIT = 1,
  K_EXPAND_OFFSETS = 2,
  K_REDUCE_RUNS = 3,
  K_MERGE_DIFF = 4,
  K_RADIX_HIST = 5,
  K_TRI_COUNT = 6,
  K_EXPAND_DENSE = 7,
  K_BS_ROUND = 8,
  K_PROV_ROUND = 9,
  K_CIRCUIT = 10,
  K_SHARD_ROUND = 11,
  K_NUM = 12,
};

inline cudaEvent_t take_event(strata_ctx* ctx) {
  if (!ctx->event_pool.empty()) {
    cudaEvent_t e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  check_cuda(cudaEventCreate(&e), "cudaEventCreate");
  return e;
}

// Returns a handle (or -1 when profiling is off); record the launch between
// kprof_begin and kprof_end.  `bytes` are the algorithmic bytes of the launch.
inline int kprof_begin(strata_ctx* ctx, int kid) {
  if (!ctx->profiling) return -1;
  strata_ctx::KRec r{kid, take_event(ctx), take_event(ctx), 0};
  check_cuda(cudaEventRecord(r.a, ctx->stream), "cudaEventRecord");
  ctx->krecs.push_back(r);
  return (int)ctx->krecs.size() - 1;
}
inline void kprof_end(strata_ctx* ctx, int h, uint64_t bytes) {
  if (h < 0) return;
  ctx->krecs[h].bytes = bytes;
  check_cuda(cudaEventRecord(ctx->krecs[h].b, ctx->stream), "cudaEventRecord");
}
// Add output bytes (known only after a count read-back) to the most recent
// record of kernel `kid`.
inline void kprof_add_last(strata_ctx* ctx, int kid, uint64_t bytes) {
  for (auto it = ctx->krecs.rbegin(); it != ctx->krecs.rend(); ++it)
    if (it->kid == kid) { it->bytes += bytes; return; }
}
// Fold finished records into the aggregates (synchronizes on the events).
inline void kprof_collect(strata_ctx* ctx) {
  for (auto& r : ctx->krecs) {
    float ms = 0;
    if (cudaEventSynchronize(r.b) == cudaSuccess && cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      auto& g = ctx->kagg[r.kid];
      g.launches++;
      g.ms += ms;
      g.bytes += r.bytes;
    }
    ctx->event_pool.push_back(r.a);
    ctx->event_pool.push_back(r.b);
  }
  ctx->krecs.clear();
}

// ---- phase timing -------------------------------------------------------------
// Records a pair of events around a phase when profiling is on and adds the
// elapsed time once the fixpoint has synchronized.
struct PhaseTimer {
  strata_ctx* ctx;
  struct Rec { cudaEvent_t a, b; double* acc; };
  std::vector<Rec> recs;
  int n = 0;
  explicit PhaseTimer(strata_ctx* c) : ctx(c) { recs.resize(4096); }
  ~PhaseTimer() {
    for (int i = 0; i < n; i++) { cudaEventDestroy(recs[i].a); cudaEventDestroy(recs[i].b); }
  }
  int begin(double* acc) {
    if (!ctx->profiling || n >= (int)recs.size()) return -1;
    Rec& r = recs[n];
    cudaEventCreate(&r.a);
    cudaEventCreate(&r.b);
    r.acc = acc;
    cudaEventRecord(r.a, ctx->stream);
    return n++;
  }
  void end(int id) {
    if (id < 0) return;
    cudaEventRecord(recs[id].b, ctx->stream);
  }
  void collect() {
    for (int i = 0; i < n; i++) {
      float ms = 0;
      if (cudaEventSynchronize(recs[i].b) == cudaSuccess &&
          cudaEventElapsedTime(&ms, recs[i].a, recs[i].b) == cudaSuccess)
        *recs[i].acc += ms;
      cudaEventDestroy(recs[i].a);
      cudaEventDestroy(recs[i].b);
    }
    n = 0;
  }
};

}  // namespace sk
