// sk_capi.cu — the extern "C" boundary declared in include/strata_b200.h.
//
// Every entry point validates its arguments, runs inside a try block that
// turns SkError into a status code (message kept in the context), and leaves
// no device work in flight when it returns.
#include "sk_ops.cuh"
#include "sk_rel.cuh"

#include <cstdlib>
#include <new>
#include <string>
#include <vector>
#include <algorithm>

using sk::DBuf;
using sk::SkError;

namespace {

#define SK_GUARD_BEGIN try {
#define SK_GUARD_END(ctx)                                                  \
  }                                                                        \
  catch (const SkError& err) {                                             \
    if (ctx) (ctx)->last_error = err.msg;                                  \
    cudaGetLastError();                                                    \
    return err.code;                                                       \
  }                                                                        \
  catch (const std::bad_alloc&) {                                          \
    if (ctx) (ctx)->last_error = "host allocation failed";                 \
    return STRATA_E_OOM;                                                   \
  }                                                                        \
  catch (...) {                                                            \
    if (ctx) (ctx)->last_error = "unexpected exception";                   \
    return STRATA_E_CUDA;                                                  \
  }                                                                        \
  return STRATA_OK;

strata_status bad(strata_ctx* ctx, const char* msg) {
  if (ctx) ctx->last_error = msg;
  return STRATA_E_INVALID;
}

template <class T>
T* host_alloc(uint64_t n) {
  void* p = std::malloc(n ? n * sizeof(T) : 1);
  if (!p) throw std::bad_alloc();
  return static_cast<T*>(p);
}

// Copy a host column to a fresh device buffer.
template <class T>
DBuf<T> to_dev(strata_ctx* ctx, const T* h, uint64_t n) {
  DBuf<T> d(ctx, n + 1);
  if (n && h) SK_CUDA(cudaMemcpyAsync(d.p, h, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  return d;
}

strata_status set_device(strata_ctx* ctx) {
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) {
    ctx->last_error = cudaGetErrorString(e);
    return STRATA_E_CUDA;
  }
  return STRATA_OK;
}

// Copy a result relation out into malloc'd host columns.
strata_status rel_out(strata_ctx* ctx, strata_rel* rel, uint32_t** os, uint32_t** od, int64_t** ow,
                      uint8_t** oi, uint64_t* on) {
  uint32_t* s = host_alloc<uint32_t>(rel->n);
  uint32_t* d = host_alloc<uint32_t>(rel->n);
  int64_t* w = ow ? host_alloc<int64_t>(rel->n) : nullptr;
  uint8_t* i = oi ? host_alloc<uint8_t>(rel->n) : nullptr;
  try {
    sk::rel_to_host(ctx, rel, s, d, w, i);
  } catch (...) {
    std::free(s); std::free(d); std::free(w); std::free(i);
    throw;
  }
  *os = s;
  *od = d;
  if (ow) *ow = w;
  if (oi) *oi = i;
  *on = rel->n;
  return STRATA_OK;
}

}  // namespace

extern "C" {

const char* strata_version(void) { return "strata-b200 0.1.0 (sm_100a)"; }

strata_status strata_ctx_create(int device, uint64_t mem_cap_bytes, strata_ctx** out) {
  if (!out) return STRATA_E_INVALID;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return STRATA_E_NOT_BUILT;
  }
  if (device < 0 || device >= count) return STRATA_E_INVALID;
  strata_ctx* ctx = new (std::nothrow) strata_ctx();
  if (!ctx) return STRATA_E_OOM;
  ctx->device = device;
  ctx->cap = mem_cap_bytes;
  SK_GUARD_BEGIN
  SK_CUDA(cudaSetDevice(device));
  SK_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  ctx->own_stream = true;
  SK_CUDA(cudaMalloc(&ctx->d_status, 256));
  SK_CUDA(cudaMemset(ctx->d_status, 0, 256));
  SK_CUDA(cudaMallocHost(&ctx->h_status, 64));
  SK_CUDA(cudaMallocHost(&ctx->h_scalar, 8 * sizeof(uint64_t)));
  SK_CUDA(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device));
  {
    // A pool of our own whose freed blocks stay mapped: per-round buffers are
    // re-used across rounds and calls instead of being re-mapped after every
    // synchronization (the default release threshold is 0).
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    SK_CUDA(cudaMemPoolCreate(&ctx->pool, &props));
    uint64_t keep = UINT64_MAX;
    SK_CUDA(cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  *out = ctx;
  }
  catch (const SkError& err) {
    cudaGetLastError();
    strata_ctx_destroy(ctx);
    return err.code;
  }
  return STRATA_OK;
}

void strata_ctx_destroy(strata_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->sizes) cudaFreeAsync(kv.first, ctx->stream);
  for (auto& kv : ctx->free_blocks) cudaFreeAsync(kv.second, ctx->stream);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->h_status) cudaFreeHost(ctx->h_status);
  if (ctx->h_scalar) cudaFreeHost(ctx->h_scalar);
  for (auto& r : ctx->krecs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
  for (auto e : ctx->event_pool) cudaEventDestroy(e);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
  delete ctx;
}

strata_status strata_ctx_set_stream(strata_ctx* ctx, void* stream) {
  if (!ctx) return STRATA_E_INVALID;
  SK_GUARD_BEGIN
  // Cached blocks were freed in the old stream's order: finish it first.
  SK_CUDA(cudaStreamSynchronize(ctx->stream));
  if (stream) {
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    ctx->stream = static_cast<cudaStream_t>(stream);
    ctx->own_stream = false;
  } else if (!ctx->own_stream) {
    SK_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->own_stream = true;
  }
  SK_GUARD_END(ctx)
}

strata_status strata_ctx_synchronize(strata_ctx* ctx) {
  if (!ctx) return STRATA_E_INVALID;
  SK_GUARD_BEGIN
  sk::sync_and_check(ctx);
  SK_GUARD_END(ctx)
}

const char* strata_last_error(const strata_ctx* ctx) {
  return ctx ? ctx->last_error.c_str() : "no context";
}

strata_status strata_ctx_mem(const strata_ctx* ctx, uint64_t* in_use, uint64_t* peak) {
  if (!ctx) return STRATA_E_INVALID;
  if (in_use) *in_use = ctx->in_use;
  if (peak) *peak = ctx->peak;
  return STRATA_OK;
}

strata_status strata_ctx_set_plan(strata_ctx* ctx, int plan) {
  if (!ctx) return STRATA_E_INVALID;
  if (plan < 0 || plan > 3)
    return bad(ctx, "plan must be 0 (auto), 1 (sort-merge), 2 (direct-addressed) or 3 (bit rows)");
  ctx->plan = plan;
  return STRATA_OK;
}

strata_status strata_ctx_set_knob(strata_ctx* ctx, int knob, int value) {
  if (!ctx) return STRATA_E_INVALID;
  if (knob == STRATA_KNOB_BATCH_GRAPH_ROUNDS) {
    if (value != 0 && value != 2 && value != 4 && value != 8 && value != 16 && value != 32)
      return bad(ctx, "graph rounds must be 0 (default), 2, 4, 8, 16 or 32");
    ctx->tune_bs_graph_rounds = value;
    return STRATA_OK;
  }
  if (knob == STRATA_KNOB_BATCH_BLOCKS_PER_SM) {
    if (value < 0 || value > 32) return bad(ctx, "blocks per SM must be 0 (default) .. 32");
    ctx->tune_bs_blocks = value;
    return STRATA_OK;
  }
  if (knob == STRATA_KNOB_BATCH_BUDGET_MB) {
    if (value < 0) return bad(ctx, "the wave budget must be >= 0 MiB");
    ctx->tune_bs_budget_mb = (uint64_t)value;
    return STRATA_OK;
  }
  if (knob == STRATA_KNOB_SORT_RANK) {
    if (value < 0 || value > 3)
      return bad(ctx, "radix ranking must be 0 (default), 1 (ballots), 2 (match) or 3 (shared masks)");
    ctx->tune_sort_rank = value == 1 ? 0 : value == 2 ? 1 : 2;
    return STRATA_OK;
  }
  if (knob == STRATA_KNOB_DENSE_WORD_MEMBERS) {
    if (value < 0 || value > 33) return bad(ctx, "dense word members must be 0 (default) .. 33");
    ctx->tune_dense_members = value;
    return STRATA_OK;
  }
  if (knob == STRATA_KNOB_WEIGHT_LANES) {
    if (value != 0 && value != 8) return bad(ctx, "weight lanes must be 0 (automatic) or 8 (always int64)");
    ctx->force_wide = value == 8;
    return STRATA_OK;
  }
  if (knob == STRATA_KNOB_TRI_PROBE) {
    if (value < 0 || value > 3)
      return bad(ctx, "triangle probe must be 0 (default), 1 (hash set), 2 (binary search) or 3 (bitmap filter)");
    ctx->tune_tri_probe = value;
    return STRATA_OK;
  }
  if (knob != STRATA_KNOB_SORT_ITEMS_U32 && knob != STRATA_KNOB_SORT_ITEMS_U64)
    return bad(ctx, "unknown knob (1 = radix keys/thread for u32 keys, 2 = for u64 keys, 3 = triangle probe)");
  const int kb = knob == STRATA_KNOB_SORT_ITEMS_U32 ? 4 : 8;
  if (value != 0) {
    int c[8];
    const int nc = sk::radix_items_choices(kb, c, 8);
    bool ok = false;
    for (int i = 0; i < nc; i++) ok |= c[i] == value;
    if (!ok) return bad(ctx, kb == 4 ? "radix keys/thread for u32 keys must be 0, 11, 15, 19 or 23"
                                     : "radix keys/thread for u64 keys must be 0, 7, 9 or 13");
  }
  (kb == 4 ? ctx->tune_items4 : ctx->tune_items8) = value;
  return STRATA_OK;
}

strata_status strata_ctx_set_profiling(strata_ctx* ctx, int enabled) {
  if (!ctx) return STRATA_E_INVALID;
  ctx->profiling = enabled != 0;
  return STRATA_OK;
}

uint64_t strata_ctx_launches(const strata_ctx* ctx) { return ctx ? ctx->launches : 0; }

strata_status strata_ctx_kernel_stats(strata_ctx* ctx, int kernel, uint64_t* launches, double* ms,
                                      uint64_t* bytes) {
  if (!ctx || kernel < 0 || kernel >= sk::K_NUM) return STRATA_E_INVALID;
  sk::kprof_collect(ctx);
  const auto& g = ctx->kagg[kernel];
  if (launches) *launches = g.launches;
  if (ms) *ms = g.ms;
  if (bytes) *bytes = g.bytes;
  return STRATA_OK;
}

strata_status strata_ctx_reset_kernel_stats(strata_ctx* ctx) {
  if (!ctx) return STRATA_E_INVALID;
  sk::kprof_collect(ctx);
  for (auto& g : ctx->kagg) g = strata_ctx::KAgg();
  return STRATA_OK;
}

void strata_free(void* p) { std::free(p); }

// ---- host-buffer drivers ---------------------------------------------------------

strata_status strata_transitive_closure_bool(strata_ctx* ctx, const uint32_t* src, const uint32_t* dst,
                                             uint64_t n, uint32_t** out_src, uint32_t** out_dst,
                                             uint64_t* out_n, strata_fix_stats* stats) {
  if (!ctx) return STRATA_E_INVALID;
  if (!out_src || !out_dst || !out_n || (n && (!src || !dst))) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  DBuf<uint32_t> ds = to_dev(ctx, src, n), dd = to_dev(ctx, dst, n);
  sk::EdgeCols e;
  e.src = ds.p; e.dst = dd.p; e.n = n;
  strata_rel* rel = sk::fix_tc_bool(ctx, e, stats);
  try {
    rel_out(ctx, rel, out_src, out_dst, nullptr, nullptr, out_n);
  } catch (...) {
    sk::rel_free(ctx, rel);
    throw;
  }
  sk::rel_free(ctx, rel);
  SK_CUDA(cudaStreamSynchronize(ctx->stream));
  SK_GUARD_END(ctx)
}

strata_status strata_shortest_paths_trop(strata_ctx* ctx, const uint32_t* src, const uint32_t* dst,
                                         const int64_t* w, const uint8_t* inf, uint64_t n,
                                         uint32_t** out_src, uint32_t** out_dst, int64_t** out_w,
                                         uint8_t** out_inf, uint64_t* out_n, strata_fix_stats* stats) {
  if (!ctx) return STRATA_E_INVALID;
  if (!out_src || !out_dst || !out_w || !out_inf || !out_n || (n && (!src || !dst || !w)))
    return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  DBuf<uint32_t> ds = to_dev(ctx, src, n), dd = to_dev(ctx, dst, n);
  DBuf<int64_t> dw = to_dev(ctx, w, n);
  DBuf<uint8_t> di;
  di.ctx = ctx;
  if (inf) di = to_dev(ctx, inf, n);
  sk::EdgeCols e;
  e.src = ds.p; e.dst = dd.p; e.w = dw.p; e.inf = inf ? di.p : nullptr; e.n = n;
  strata_rel* rel = sk::fix_trop_paths(ctx, e, stats);
  try {
    rel_out(ctx, rel, out_src, out_dst, out_w, out_inf, out_n);
  } catch (...) {
    sk::rel_free(ctx, rel);
    throw;
  }
  sk::rel_free(ctx, rel);
  SK_CUDA(cudaStreamSynchronize(ctx->stream));
  SK_GUARD_END(ctx)
}

strata_status strata_mssp_trop(strata_ctx* ctx, const uint32_t* sources, const int64_t* src_w,
                               const uint8_t* src_inf, uint64_t ns, const uint32_t* esrc,
                               const uint32_t* edst, const int64_t* ew, const uint8_t* einf,
                               uint64_t ne, uint32_t** out_src, uint32_t** out_dst, int64_t** out_w,
                               uint8_t** out_inf, uint64_t* out_n, strata_fix_stats* stats) {
  if (!ctx) return STRATA_E_INVALID;
  if (!out_src || !out_dst || !out_w || !out_inf || !out_n || (ns && !sources) ||
      (ne && (!esrc || !edst || !ew)))
    return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  DBuf<uint32_t> dsrc = to_dev(ctx, sources, ns);
  DBuf<int64_t> dsw;
  DBuf<uint8_t> dsi, dei;
  dsw.ctx = dsi.ctx = dei.ctx = ctx;
  if (src_w) dsw = to_dev(ctx, src_w, ns);
  if (src_inf) dsi = to_dev(ctx, src_inf, ns);
  DBuf<uint32_t> ds = to_dev(ctx, esrc, ne), dd = to_dev(ctx, edst, ne);
  DBuf<int64_t> dw = to_dev(ctx, ew, ne);
  if (einf) dei = to_dev(ctx, einf, ne);
  sk::EdgeCols e;
  e.src = ds.p; e.dst = dd.p; e.w = dw.p; e.inf = einf ? dei.p : nullptr; e.n = ne;
  strata_rel* rel = sk::fix_mssp(ctx, dsrc.p, src_w ? dsw.p : nullptr, src_inf ? dsi.p : nullptr, ns, e, stats);
  try {
    rel_out(ctx, rel, out_src, out_dst, out_w, out_inf, out_n);
  } catch (...) {
    sk::rel_free(ctx, rel);
    throw;
  }
  sk::rel_free(ctx, rel);
  SK_CUDA(cudaStreamSynchronize(ctx->stream));
  SK_GUARD_END(ctx)
}

#define SK_COUNT_ENTRY(NAME, FN)                                                            \
  strata_status NAME(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n,     \
                     uint64_t* out) {                                                       \
    if (!ctx) return STRATA_E_INVALID;                                                      \
    if (!out || (n && (!a || !b))) return bad(ctx, "NULL argument");                        \
    if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;                                 \
    SK_GUARD_BEGIN                                                                          \
    DBuf<uint32_t> da = to_dev(ctx, a, n), db = to_dev(ctx, b, n);                          \
    *out = FN(ctx, da.p, db.p, n);                                                          \
    SK_CUDA(cudaStreamSynchronize(ctx->stream));                                            \
    SK_GUARD_END(ctx)                                                                       \
  }

SK_COUNT_ENTRY(strata_count_triangles, sk::count_triangles_undirected)
SK_COUNT_ENTRY(strata_count_4cliques, sk::count_4cliques_undirected)
SK_COUNT_ENTRY(strata_count_triangle_pattern, sk::count_triangle_pattern)
SK_COUNT_ENTRY(strata_binary_plan_intermediate, sk::binary_plan_intermediate)
#undef SK_COUNT_ENTRY

strata_status strata_intern_terms(strata_ctx* ctx, const uint64_t* keys, uint64_t n, uint32_t* ids_out,
                                  uint64_t* n_distinct) {
  if (!ctx) return STRATA_E_INVALID;
  if ((n && (!keys || !ids_out))) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  DBuf<uint64_t> dk = to_dev(ctx, keys, n);
  DBuf<uint32_t> di(ctx, n + 1);
  const uint64_t m = sk::intern_terms(ctx, dk.p, n, di.p);
  if (n) SK_CUDA(cudaMemcpyAsync(ids_out, di.p, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  SK_CUDA(cudaStreamSynchronize(ctx->stream));
  if (n_distinct) *n_distinct = m;
  SK_GUARD_END(ctx)
}

// ---- device-resident drivers ------------------------------------------------------

strata_status strata_tc_bool_dev(strata_ctx* ctx, const uint32_t* d_src, const uint32_t* d_dst, uint64_t n,
                                 strata_rel** out, strata_fix_stats* stats) {
  if (!ctx) return STRATA_E_INVALID;
  if (!out || (n && (!d_src || !d_dst))) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::EdgeCols e;
  e.src = d_src; e.dst = d_dst; e.n = n;
  *out = sk::fix_tc_bool(ctx, e, stats);
  SK_GUARD_END(ctx)
}

strata_status strata_trop_paths_dev(strata_ctx* ctx, const uint32_t* d_src, const uint32_t* d_dst,
                                    const int64_t* d_w, const uint8_t* d_inf, uint64_t n, strata_rel** out,
                                    strata_fix_stats* stats) {
  if (!ctx) return STRATA_E_INVALID;
  if (!out || (n && (!d_src || !d_dst || !d_w))) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::EdgeCols e;
  e.src = d_src; e.dst = d_dst; e.w = d_w; e.inf = d_inf; e.n = n;
  *out = sk::fix_trop_paths(ctx, e, stats);
  SK_GUARD_END(ctx)
}

strata_status strata_mssp_trop_dev(strata_ctx* ctx, const uint32_t* d_sources, const int64_t* d_src_w,
                                   const uint8_t* d_src_inf, uint64_t ns, const uint32_t* d_esrc,
                                   const uint32_t* d_edst, const int64_t* d_ew, const uint8_t* d_einf,
                                   uint64_t ne, strata_rel** out, strata_fix_stats* stats) {
  if (!ctx) return STRATA_E_INVALID;
  if (!out || (ns && !d_sources) || (ne && (!d_esrc || !d_edst || !d_ew))) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::EdgeCols e;
  e.src = d_esrc; e.dst = d_edst; e.w = d_ew; e.inf = d_einf; e.n = ne;
  *out = sk::fix_mssp(ctx, d_sources, d_src_w, d_src_inf, ns, e, stats);
  SK_GUARD_END(ctx)
}

strata_status strata_count_triangle_pattern_dev(strata_ctx* ctx, const uint32_t* d_x, const uint32_t* d_y,
                                                uint64_t n, uint64_t* out_count) {
  if (!ctx) return STRATA_E_INVALID;
  if (!out_count || (n && (!d_x || !d_y))) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  *out_count = sk::count_triangle_pattern(ctx, d_x, d_y, n);
  SK_GUARD_END(ctx)
}

// ---- batched Bool reachability -----------------------------------------------------

namespace {
strata_status batch_check(strata_ctx* ctx, uint32_t n_inst, const uint32_t* nodes, const uint64_t* edge_off,
                          const void* src, const void* dst) {
  if (n_inst && (!nodes || !edge_off)) return bad(ctx, "NULL argument");
  if (n_inst && edge_off[0] != 0) return bad(ctx, "edge_off[0] must be 0");
  for (uint32_t i = 0; i < n_inst; i++)
    if (edge_off[i + 1] < edge_off[i]) return bad(ctx, "edge offsets must be non-decreasing");
  if (n_inst && edge_off[n_inst] && (!src || !dst)) return bad(ctx, "NULL argument");
  return STRATA_OK;
}
}  // namespace

strata_status strata_tc_bool_batch_dev(strata_ctx* ctx, uint32_t n_inst, const uint32_t* nodes,
                                       const uint64_t* edge_off, const uint32_t* d_src, const uint32_t* d_dst,
                                       int mode, uint64_t* counts, uint64_t* fps, uint32_t* rounds,
                                       strata_batch_stats* stats) {
  if (!ctx) return STRATA_E_INVALID;
  if (batch_check(ctx, n_inst, nodes, edge_off, d_src, d_dst) != STRATA_OK) return STRATA_E_INVALID;
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::tc_bool_batch(ctx, n_inst, nodes, edge_off, d_src, d_dst, mode, counts, fps, rounds, stats);
  SK_GUARD_END(ctx)
}

strata_status strata_tc_bool_batch(strata_ctx* ctx, uint32_t n_inst, const uint32_t* nodes,
                                   const uint64_t* edge_off, const uint32_t* src, const uint32_t* dst, int mode,
                                   uint64_t* counts, uint64_t* fps, uint32_t* rounds, strata_batch_stats* stats) {
  if (!ctx) return STRATA_E_INVALID;
  if (batch_check(ctx, n_inst, nodes, edge_off, src, dst) != STRATA_OK) return STRATA_E_INVALID;
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  const uint64_t m = n_inst ? edge_off[n_inst] : 0;
  DBuf<uint32_t> ds = to_dev(ctx, src, m), dd = to_dev(ctx, dst, m);
  sk::tc_bool_batch(ctx, n_inst, nodes, edge_off, ds.p, dd.p, mode, counts, fps, rounds, stats);
  SK_GUARD_END(ctx)
}

// ---- sharded Bool closure -------------------------------------------------------

strata_status strata_tc_shard_create(strata_ctx* ctx, uint32_t n_nodes, const uint32_t* d_src,
                                     const uint32_t* d_dst, uint64_t m, uint32_t rank, uint32_t world,
                                     strata_tc_shard** out) {
  if (!ctx || !out) return STRATA_E_INVALID;
  *out = nullptr;
  if (world == 0 || rank >= world || n_nodes == 0) return bad(ctx, "need world >= 1, rank < world and n_nodes >= 1");
  if (m && (!d_src || !d_dst)) return bad(ctx, "null edge columns");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  auto* sh = new strata_tc_shard();
  sh->ctx = ctx;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  sk::tc_shard_init(ctx, sh, n_nodes, d_src, d_dst, m, rank, world);
  *out = sh;
  return STRATA_OK;
  }
  catch (const SkError& err) {
    delete sh;
    ctx->last_error = err.msg;
    cudaGetLastError();
    return err.code;
  }
  catch (...) {
    delete sh;
    return STRATA_E_CUDA;
  }
}

strata_status strata_tc_shard_shape(const strata_tc_shard* sh, uint32_t* rows_per_rank, uint32_t* row_lo,
                                    uint32_t* row_hi, uint64_t* row_bytes) {
  if (!sh) return STRATA_E_INVALID;
  if (rows_per_rank) *rows_per_rank = sh->per;
  if (row_lo) *row_lo = sh->lo;
  if (row_hi) *row_hi = sh->hi;
  if (row_bytes) *row_bytes = (uint64_t)sh->w4 * 16;
  return STRATA_OK;
}

strata_status strata_tc_shard_seed(strata_ctx* ctx, strata_tc_shard* sh, void* d_delta_mine, uint8_t* d_flags_mine,
                                   uint64_t* n_delta) {
  if (!ctx || !sh || sh->ctx != ctx || !d_delta_mine || !d_flags_mine) return STRATA_E_INVALID;
  if (reinterpret_cast<uintptr_t>(d_delta_mine) % 16) return bad(ctx, "the Delta slice must be 16-byte aligned");
  if (sh->seeded) return bad(ctx, "the share is already seeded (its edge columns were released)");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  const uint64_t c = sk::tc_shard_seed(ctx, sh, static_cast<uint4*>(d_delta_mine), d_flags_mine);
  if (n_delta) *n_delta = c;
  SK_GUARD_END(ctx)
}

strata_status strata_tc_shard_round(strata_ctx* ctx, strata_tc_shard* sh, const void* d_delta_full,
                                    const uint8_t* d_flags_full, void* d_delta_mine, uint8_t* d_flags_mine,
                                    uint64_t* n_delta) {
  if (!ctx || !sh || sh->ctx != ctx || !d_delta_full || !d_flags_full || !d_delta_mine || !d_flags_mine)
    return STRATA_E_INVALID;
  if (reinterpret_cast<uintptr_t>(d_delta_full) % 16 || reinterpret_cast<uintptr_t>(d_delta_mine) % 16)
    return bad(ctx, "Delta buffers must be 16-byte aligned");
  const uint64_t full_bytes = (uint64_t)sh->world * sh->per * sh->w4 * 16;
  const auto f0 = reinterpret_cast<uintptr_t>(d_delta_full), m0 = reinterpret_cast<uintptr_t>(d_delta_mine);
  const uint64_t mine_bytes = (uint64_t)sh->per * sh->w4 * 16;
  if (m0 < f0 + full_bytes && f0 < m0 + mine_bytes) return bad(ctx, "the Delta slice overlaps the gathered Delta");
  const auto g0 = reinterpret_cast<uintptr_t>(d_flags_full), h0 = reinterpret_cast<uintptr_t>(d_flags_mine);
  const uint64_t gfull = (uint64_t)sh->world * sh->per, gmine = sh->per;
  if (h0 < g0 + gfull && g0 < h0 + gmine) return bad(ctx, "the row flags slice overlaps the gathered row flags");
  if (!sh->seeded) return bad(ctx, "round before seed: call strata_tc_shard_seed first");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  const uint64_t c = sk::tc_shard_round(ctx, sh, static_cast<const uint4*>(d_delta_full), d_flags_full,
                                        static_cast<uint4*>(d_delta_mine), d_flags_mine);
  if (n_delta) *n_delta = c;
  SK_GUARD_END(ctx)
}

strata_status strata_tc_shard_pack(strata_ctx* ctx, strata_tc_shard* sh, const void* d_delta_mine,
                                   int64_t* d_out, uint64_t cap, uint64_t* n_words) {
  if (!ctx || !sh || sh->ctx != ctx || !d_delta_mine || !n_words || (cap && !d_out)) return STRATA_E_INVALID;
  if (reinterpret_cast<uintptr_t>(d_delta_mine) % 16) return bad(ctx, "Delta buffers must be 16-byte aligned");
  if (!sh->seeded) return bad(ctx, "pack before seed: call strata_tc_shard_seed first");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  *n_words = sk::tc_shard_pack(ctx, sh, static_cast<const uint4*>(d_delta_mine), d_out, cap);
  SK_GUARD_END(ctx)
}

strata_status strata_tc_shard_unpack(strata_ctx* ctx, strata_tc_shard* sh, const int64_t* d_in, uint64_t n,
                                     void* d_delta_full, uint8_t* d_flags_full) {
  if (!ctx || !sh || sh->ctx != ctx || !d_delta_full || !d_flags_full || (n && !d_in)) return STRATA_E_INVALID;
  if (reinterpret_cast<uintptr_t>(d_delta_full) % 16) return bad(ctx, "Delta buffers must be 16-byte aligned");
  const uint64_t full_bytes = (uint64_t)sh->world * sh->per * sh->w4 * 16;
  const auto f0 = reinterpret_cast<uintptr_t>(d_delta_full), i0 = reinterpret_cast<uintptr_t>(d_in);
  if (n && i0 < f0 + full_bytes && f0 < i0 + n * 24) return bad(ctx, "the packed words overlap the gathered Delta");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  sk::tc_shard_unpack(ctx, sh, d_in, n, static_cast<uint4*>(d_delta_full), d_flags_full);
  SK_GUARD_END(ctx)
}

strata_status strata_tc_shard_summary(strata_ctx* ctx, strata_tc_shard* sh, uint64_t* count, uint64_t* fingerprint) {
  if (!ctx || !sh || sh->ctx != ctx) return STRATA_E_INVALID;
  if (!sh->seeded) return bad(ctx, "summary before seed: call strata_tc_shard_seed first");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  uint64_t c, f;
  sk::tc_shard_summary(ctx, sh, &c, &f);
  if (count) *count = c;
  if (fingerprint) *fingerprint = f;
  SK_GUARD_END(ctx)
}

void strata_tc_shard_free(strata_tc_shard* sh) {
  if (!sh) return;
  try {
    delete sh;  // device buffers go back to the context's pool
  } catch (...) {
  }
}

// ---- Prov_k capture and provenance circuits --------------------------------------

struct strata_proofs {
  std::vector<std::vector<std::vector<uint32_t>>> q;
};

strata_status strata_prov_tc_capture(strata_ctx* ctx, uint32_t n_nodes, const uint32_t* d_src,
                                     const uint32_t* d_dst, uint64_t n_edges, const double* d_prob, uint32_t k,
                                     uint32_t n_queries, const uint32_t* qs, const uint32_t* qt,
                                     strata_proofs** out, uint32_t* target_rounds, strata_prov_stats* stats) {
  if (!ctx) return STRATA_E_INVALID;
  if (!out || (n_edges && (!d_src || !d_dst || !d_prob)) || (n_queries && (!qs || !qt)))
    return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  auto* pr = new strata_proofs();
  std::vector<uint32_t> rounds;
  try {
    sk::prov_tc_capture(ctx, n_nodes, d_src, d_dst, n_edges, d_prob, k, n_queries, qs, qt, pr->q, rounds, stats);
  } catch (...) {
    delete pr;
    throw;
  }
  if (target_rounds) std::copy(rounds.begin(), rounds.end(), target_rounds);
  *out = pr;
  SK_GUARD_END(ctx)
}

strata_status strata_proofs_shape(const strata_proofs* pr, uint32_t* n_queries, uint64_t* n_proofs,
                                  uint64_t* n_lits) {
  if (!pr) return STRATA_E_INVALID;
  uint64_t np = 0, nl = 0;
  for (auto& q : pr->q) {
    np += q.size();
    for (auto& p : q) nl += p.size();
  }
  if (n_queries) *n_queries = (uint32_t)pr->q.size();
  if (n_proofs) *n_proofs = np;
  if (n_lits) *n_lits = nl;
  return STRATA_OK;
}

strata_status strata_proofs_export(const strata_proofs* pr, uint64_t* proof_off, uint64_t* lit_off, int64_t* lits) {
  if (!pr || !proof_off || !lit_off) return STRATA_E_INVALID;
  uint64_t np = 0, nl = 0;
  for (size_t q = 0; q < pr->q.size(); q++) {
    proof_off[q] = np;
    for (auto& p : pr->q[q]) {
      lit_off[np++] = nl;
      for (auto l : p) {
        if (lits) lits[nl] = (int64_t)l;
        nl++;
      }
    }
  }
  proof_off[pr->q.size()] = np;
  lit_off[np] = nl;
  return STRATA_OK;
}

void strata_proofs_free(strata_proofs* pr) { delete pr; }

strata_status strata_circuits_compile(strata_ctx* ctx, uint32_t n_queries, const uint64_t* proof_off,
                                      const uint64_t* lit_off, const int64_t* lits, uint32_t n_leaves,
                                      uint64_t max_nodes, strata_circuits** out) {
  if (!ctx) return STRATA_E_INVALID;
  if (!out || (n_queries && (!proof_off || !lit_off))) return bad(ctx, "NULL argument");
  if (n_queries && lit_off[proof_off[n_queries]] && !lits) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  *out = sk::circuits_compile(ctx, n_queries, proof_off, lit_off, lits, n_leaves, max_nodes ? max_nodes : (1u << 20));
  SK_GUARD_END(ctx)
}

struct strata_circuit_parts {
  sk::CircuitParts* p = nullptr;
};

namespace {
thread_local std::string g_parts_error;
}

strata_status strata_circuits_compile_host(uint32_t n_queries, const uint64_t* proof_off, const uint64_t* lit_off,
                                           const int64_t* lits, uint32_t n_leaves, uint64_t max_nodes,
                                           strata_circuit_parts** out) {
  if (!out || (n_queries && (!proof_off || !lit_off))) {
    g_parts_error = "NULL argument";
    return STRATA_E_INVALID;
  }
  if (n_queries && lit_off[proof_off[n_queries]] && !lits) {
    g_parts_error = "NULL argument";
    return STRATA_E_INVALID;
  }
  try {
    auto* h = new strata_circuit_parts();
    try {
      h->p = sk::circuit_parts_compile(n_queries, proof_off, lit_off, lits, n_leaves,
                                       max_nodes ? max_nodes : (1u << 20));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return STRATA_OK;
  } catch (const SkError& err) {
    g_parts_error = err.msg;
    return err.code;
  } catch (const std::bad_alloc&) {
    g_parts_error = "host allocation failed";
    return STRATA_E_OOM;
  } catch (...) {
    g_parts_error = "unexpected exception";
    return STRATA_E_CUDA;
  }
}

const char* strata_circuit_parts_error(void) { return g_parts_error.c_str(); }

strata_status strata_circuits_upload(strata_ctx* ctx, uint32_t n_parts, strata_circuit_parts* const* parts,
                                     uint32_t n_leaves, strata_circuits** out) {
  if (!ctx) return STRATA_E_INVALID;
  if (!out || (n_parts && !parts)) return bad(ctx, "NULL argument");
  for (uint32_t i = 0; i < n_parts; i++)
    if (!parts[i] || !parts[i]->p) return bad(ctx, "NULL part");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  std::vector<sk::CircuitParts*> v;
  for (uint32_t i = 0; i < n_parts; i++) v.push_back(parts[i]->p);
  *out = sk::circuit_parts_upload(ctx, n_parts, v.data(), n_leaves);
  SK_GUARD_END(ctx)
}

void strata_circuit_parts_free(strata_circuit_parts* parts) {
  if (!parts) return;
  sk::circuit_parts_free(parts->p);
  delete parts;
}

strata_status strata_circuit_parts_shape(const strata_circuit_parts* parts, uint32_t* n_queries, uint64_t* n_nodes,
                                        uint32_t* max_levels) {
  if (!parts || !parts->p) return STRATA_E_INVALID;
  const uint64_t n = sk::circuit_parts_nodes(parts->p, max_levels);
  if (n_nodes) *n_nodes = n;
  if (n_queries) *n_queries = sk::circuit_parts_queries(parts->p);
  return STRATA_OK;
}

strata_status strata_circuit_parts_eval64(const strata_circuit_parts* parts, const double* prob, double* out) {
  if (!parts || !parts->p || !out) return STRATA_E_INVALID;
  sk::circuit_parts_eval64(parts->p, prob, out);
  return STRATA_OK;
}

strata_status strata_circuits_shape(const strata_circuits* c, uint64_t* n_nodes, uint32_t* max_levels) {
  if (!c) return STRATA_E_INVALID;
  if (n_nodes) *n_nodes = c->n_nodes;
  if (max_levels) *max_levels = c->max_levels;
  return STRATA_OK;
}

strata_status strata_circuits_forward(strata_ctx* ctx, const strata_circuits* c, const float* d_p, float* d_out,
                                      double* d_out64) {
  if (!ctx) return STRATA_E_INVALID;
  if (!c || (c->n_leaves && !d_p) || (!d_out && !d_out64)) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::circuits_forward(ctx, c, d_p, d_out, d_out64);
  SK_GUARD_END(ctx)
}

strata_status strata_circuits_vjp(strata_ctx* ctx, const strata_circuits* c, const float* d_p, const float* d_seed,
                                  double* d_grad64, float* d_grad32) {
  if (!ctx) return STRATA_E_INVALID;
  if (!c || (c->n_leaves && (!d_p || !d_grad64))) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::circuits_adjoint(ctx, c, d_p, d_seed, d_grad64, 0, d_grad32);
  SK_GUARD_END(ctx)
}

strata_status strata_circuits_grads(strata_ctx* ctx, const strata_circuits* c, const float* d_p, double* d_grads) {
  if (!ctx) return STRATA_E_INVALID;
  if (!c || (c->n_leaves && c->n_queries && (!d_p || !d_grads))) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::circuits_adjoint(ctx, c, d_p, nullptr, d_grads, 1, nullptr);
  SK_GUARD_END(ctx)
}

void strata_circuits_free(strata_ctx* ctx, strata_circuits* c) {
  if (!ctx || !c) return;
  try {
    sk::circuits_free(ctx, c);
  } catch (...) {
  }
}

strata_status strata_count_triangle_pattern_range_dev(strata_ctx* ctx, const uint32_t* d_x, const uint32_t* d_y,
                                                      uint64_t n, uint64_t x_lo, uint64_t x_hi,
                                                      uint64_t* out_count) {
  if (!ctx) return STRATA_E_INVALID;
  if (!out_count || (n && (!d_x || !d_y))) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  *out_count = sk::count_triangle_pattern_range(ctx, d_x, d_y, n, x_lo, x_hi);
  SK_GUARD_END(ctx)
}

strata_status strata_rel_size(const strata_rel* rel, uint64_t* n) {
  if (!rel || !n) return STRATA_E_INVALID;
  *n = rel->n;
  return STRATA_OK;
}

strata_status strata_rel_is_trop(const strata_rel* rel, int* is_trop) {
  if (!rel || !is_trop) return STRATA_E_INVALID;
  *is_trop = rel->trop ? 1 : 0;
  return STRATA_OK;
}

strata_status strata_rel_to_host(strata_ctx* ctx, const strata_rel* rel, uint32_t* src, uint32_t* dst,
                                 int64_t* w, uint8_t* inf) {
  if (!ctx || !rel) return STRATA_E_INVALID;
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::rel_to_host(ctx, rel, src, dst, w, inf);
  SK_GUARD_END(ctx)
}

strata_status strata_rel_fingerprint(strata_ctx* ctx, const strata_rel* rel, uint64_t* fp) {
  if (!ctx || !rel || !fp) return STRATA_E_INVALID;
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  *fp = sk::rel_fingerprint(ctx, rel);
  SK_GUARD_END(ctx)
}

void strata_rel_free(strata_ctx* ctx, strata_rel* rel) {
  if (ctx) cudaSetDevice(ctx->device);
  sk::rel_free(ctx, rel);
}

// ---- operator surface ---------------------------------------------------------------

strata_status strata_op_sort(strata_ctx* ctx, int key_bytes, int val_bytes, const void* d_keys_in,
                             const void* d_vals_in, void* d_keys_out, void* d_vals_out, uint64_t n,
                             int key_bits) {
  if (!ctx) return STRATA_E_INVALID;
  if ((key_bytes != 4 && key_bytes != 8) || (val_bytes != 0 && val_bytes != 4 && val_bytes != 8))
    return bad(ctx, "key_bytes must be 4 or 8, val_bytes 0, 4 or 8");
  if (n && (!d_keys_in || !d_keys_out || (val_bytes && (!d_vals_in || !d_vals_out))))
    return bad(ctx, "NULL argument");
  if (key_bits < 0 || key_bits > 8 * key_bytes) return bad(ctx, "key_bits out of range");
  if (n > sk::kMaxSortKeys) return bad(ctx, "n exceeds 2^32-1");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  if (n == 0) return STRATA_OK;
  // Copy the inputs into the output buffers, sort between output and scratch.
  SK_CUDA(cudaMemcpyAsync(d_keys_out, d_keys_in, n * key_bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  if (val_bytes)
    SK_CUDA(cudaMemcpyAsync(d_vals_out, d_vals_in, n * val_bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  auto run = [&](auto kt, auto vt) {
    using K = decltype(kt);
    using V = decltype(vt);
    DBuf<K> ka(ctx, n);
    DBuf<V> va;
    va.ctx = ctx;
    if (val_bytes) va.reserve(n);
    K* kp = static_cast<K*>(d_keys_out);
    K* kalt = ka.p;
    V* vp = static_cast<V*>(d_vals_out);
    V* valt = va.p;
    sk::radix_sort<K, V>(ctx, &kp, &kalt, &vp, &valt, val_bytes != 0, n, key_bits, true);
    if (kp != d_keys_out) {
      SK_CUDA(cudaMemcpyAsync(d_keys_out, kp, n * sizeof(K), cudaMemcpyDeviceToDevice, ctx->stream));
      if (val_bytes) SK_CUDA(cudaMemcpyAsync(d_vals_out, vp, n * sizeof(V), cudaMemcpyDeviceToDevice, ctx->stream));
    }
    sk::sync_and_check(ctx);
  };
  if (key_bytes == 4) {
    if (val_bytes == 8) run(uint32_t(), uint64_t()); else run(uint32_t(), uint32_t());
  } else {
    if (val_bytes == 8) run(uint64_t(), uint64_t()); else run(uint64_t(), uint32_t());
  }
  SK_GUARD_END(ctx)
}

// [a, a + an) and [b, b + bn) share a byte (null or empty spans share none).
static bool spans_overlap(const void* a, uint64_t an, const void* b, uint64_t bn) {
  const auto x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return a && b && an && bn && x < y + bn && y < x + an;
}

strata_status strata_op_dedup_diff(strata_ctx* ctx, int key_bytes, const void* d_cand, uint64_t n,
                                   const void* d_full, uint64_t n_full, void* d_out, uint64_t* out_n) {
  if (!ctx) return STRATA_E_INVALID;
  if (key_bytes != 4 && key_bytes != 8) return bad(ctx, "key_bytes must be 4 or 8");
  if (!out_n || (n && (!d_cand || !d_out)) || (n_full && !d_full)) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  DBuf<uint64_t> cnt(ctx, 1);
  if (key_bytes == 4)
    sk::diff_improve<uint32_t, int32_t, false>(ctx, (const uint32_t*)d_cand, nullptr, n, (const uint32_t*)d_full,
                                               nullptr, n_full, (uint32_t*)d_out, nullptr, cnt.p);
  else
    sk::diff_improve<uint64_t, int32_t, false>(ctx, (const uint64_t*)d_cand, nullptr, n, (const uint64_t*)d_full,
                                               nullptr, n_full, (uint64_t*)d_out, nullptr, cnt.p);
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, cnt.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
  sk::sync_and_check(ctx);
  *out_n = ctx->h_scalar[0];
  SK_GUARD_END(ctx)
}

strata_status strata_op_min_improve(strata_ctx* ctx, int key_bytes, const void* d_cand, const int64_t* d_cand_w,
                                    uint64_t n, const void* d_full, int64_t* d_full_w, uint64_t n_full,
                                    void* d_out_keys, int64_t* d_out_w, uint64_t* out_n) {
  if (!ctx) return STRATA_E_INVALID;
  if (key_bytes != 4 && key_bytes != 8) return bad(ctx, "key_bytes must be 4 or 8");
  if (!out_n || (n && (!d_cand || !d_cand_w || !d_out_keys || !d_out_w)) || (n_full && (!d_full || !d_full_w)))
    return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  DBuf<uint64_t> cnt(ctx, 1);
  if (key_bytes == 4)
    sk::diff_improve<uint32_t, int64_t, true>(ctx, (const uint32_t*)d_cand, d_cand_w, n, (const uint32_t*)d_full,
                                              d_full_w, n_full, (uint32_t*)d_out_keys, d_out_w, cnt.p);
  else
    sk::diff_improve<uint64_t, int64_t, true>(ctx, (const uint64_t*)d_cand, d_cand_w, n, (const uint64_t*)d_full,
                                              d_full_w, n_full, (uint64_t*)d_out_keys, d_out_w, cnt.p);
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, cnt.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
  sk::sync_and_check(ctx);
  *out_n = ctx->h_scalar[0];
  SK_GUARD_END(ctx)
}

strata_status strata_op_reduce(strata_ctx* ctx, int key_bytes, const void* d_keys, const int64_t* d_w, uint64_t n,
                               void* d_out, int64_t* d_out_w, uint64_t* out_n) {
  if (!ctx) return STRATA_E_INVALID;
  if (key_bytes != 4 && key_bytes != 8) return bad(ctx, "key_bytes must be 4 or 8");
  if (!out_n || (n && (!d_keys || !d_out || (d_w && !d_out_w)))) return bad(ctx, "NULL argument");
  if (n > sk::kMaxSortN) return bad(ctx, "n is limited to 2^30 - 1 per call");
  {
    // tiles write their output while other tiles still read their input
    const uint64_t kb = n * (uint64_t)key_bytes, wb = n * 8;
    if (spans_overlap(d_keys, kb, d_out, kb) || spans_overlap(d_keys, kb, d_out_w, wb) ||
        spans_overlap(d_w, wb, d_out, kb) || spans_overlap(d_w, wb, d_out_w, wb))
      return bad(ctx, "the output buffers overlap the input buffers");
  }
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  DBuf<uint64_t> cnt(ctx, 1);
  if (key_bytes == 4) {
    if (d_w) sk::reduce_runs<uint32_t, int64_t, true>(ctx, (const uint32_t*)d_keys, d_w, n, (uint32_t*)d_out, d_out_w, cnt.p);
    else sk::reduce_runs<uint32_t, int32_t, false>(ctx, (const uint32_t*)d_keys, nullptr, n, (uint32_t*)d_out, nullptr, cnt.p);
  } else {
    if (d_w) sk::reduce_runs<uint64_t, int64_t, true>(ctx, (const uint64_t*)d_keys, d_w, n, (uint64_t*)d_out, d_out_w, cnt.p);
    else sk::reduce_runs<uint64_t, int32_t, false>(ctx, (const uint64_t*)d_keys, nullptr, n, (uint64_t*)d_out, nullptr, cnt.p);
  }
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, cnt.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
  sk::sync_and_check(ctx);
  *out_n = ctx->h_scalar[0];
  SK_GUARD_END(ctx)
}

strata_status strata_op_merge_diff(strata_ctx* ctx, int key_bytes, const void* d_full, const int64_t* d_full_w,
                                   uint64_t n_full, const void* d_cand, const int64_t* d_cand_w, uint64_t n_cand,
                                   void* d_full_out, int64_t* d_full_out_w, void* d_delta, int64_t* d_delta_w,
                                   uint64_t* out_full_n, uint64_t* out_delta_n) {
  if (!ctx) return STRATA_E_INVALID;
  if (key_bytes != 4 && key_bytes != 8) return bad(ctx, "key_bytes must be 4 or 8");
  const bool trop = d_cand_w != nullptr;
  if (!out_full_n || !out_delta_n || (n_full && !d_full) || (n_cand && !d_cand) || !d_full_out || !d_delta)
    return bad(ctx, "NULL argument");
  if (trop && ((n_full && !d_full_w) || !d_full_out_w || !d_delta_w)) return bad(ctx, "NULL weight column");
  if (n_full + n_cand > sk::kMaxSortN) return bad(ctx, "n is limited to 2^30 - 1 per call");
  {
    // tiles write their output while other tiles still read their input
    const uint64_t kb = key_bytes, fo = n_full + n_cand;
    const void* in[4] = {d_full, d_full_w, d_cand, d_cand_w};
    const uint64_t in_b[4] = {n_full * kb, n_full * 8, n_cand * kb, n_cand * 8};
    const void* out[4] = {d_full_out, d_full_out_w, d_delta, d_delta_w};
    const uint64_t out_b[4] = {fo * kb, fo * 8, n_cand * kb, n_cand * 8};
    for (int a = 0; a < 4; a++)
      for (int b = 0; b < 4; b++)
        if (spans_overlap(in[a], in_b[a], out[b], out_b[b]))
          return bad(ctx, "the output buffers overlap the input buffers");
  }
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  DBuf<uint64_t> cnt(ctx, 2);
  if (key_bytes == 4) {
    if (trop) sk::merge_diff<uint32_t, int64_t, true>(ctx, (const uint32_t*)d_full, d_full_w, n_full, (const uint32_t*)d_cand,
                                                      d_cand_w, n_cand, (uint32_t*)d_full_out, d_full_out_w,
                                                      (uint32_t*)d_delta, d_delta_w, cnt.p);
    else sk::merge_diff<uint32_t, int32_t, false>(ctx, (const uint32_t*)d_full, nullptr, n_full, (const uint32_t*)d_cand,
                                                  nullptr, n_cand, (uint32_t*)d_full_out, nullptr, (uint32_t*)d_delta,
                                                  nullptr, cnt.p);
  } else {
    if (trop) sk::merge_diff<uint64_t, int64_t, true>(ctx, (const uint64_t*)d_full, d_full_w, n_full, (const uint64_t*)d_cand,
                                                      d_cand_w, n_cand, (uint64_t*)d_full_out, d_full_out_w,
                                                      (uint64_t*)d_delta, d_delta_w, cnt.p);
    else sk::merge_diff<uint64_t, int32_t, false>(ctx, (const uint64_t*)d_full, nullptr, n_full, (const uint64_t*)d_cand,
                                                  nullptr, n_cand, (uint64_t*)d_full_out, nullptr, (uint64_t*)d_delta,
                                                  nullptr, cnt.p);
  }
  SK_CUDA(cudaMemcpyAsync(ctx->h_scalar, cnt.p, 16, cudaMemcpyDeviceToHost, ctx->stream));
  sk::sync_and_check(ctx);
  *out_full_n = ctx->h_scalar[0];
  *out_delta_n = ctx->h_scalar[1];
  SK_GUARD_END(ctx)
}

strata_status strata_asp_simplify_filter(strata_ctx* ctx, uint64_t n_rules, const int32_t* head,
                                         const uint32_t* body_start, const int32_t* body_lit, uint64_t n_atoms,
                                         const uint8_t* poss, const uint8_t* cert, int32_t** out_head,
                                         uint32_t** out_body_start, int32_t** out_body_lit, uint64_t* out_n) {
  if (!ctx) return STRATA_E_INVALID;
  if (!out_head || !out_body_start || !out_body_lit || !out_n || (n_rules && (!head || !body_start)) ||
      (n_atoms && (!poss || !cert)))
    return bad(ctx, "NULL argument");
  if (n_rules && body_start[n_rules] && !body_lit) return bad(ctx, "NULL body literals");
  if (n_rules >= 0xffffffffull) return bad(ctx, "at most 2^32 - 2 rules per call");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  sk::AspResult r = sk::asp_simplify(ctx, n_rules, head, body_start, body_lit, n_atoms, poss, cert);
  *out_head = r.head;
  *out_body_start = r.body_start;
  *out_body_lit = r.body_lit;
  *out_n = r.n_rules;
  SK_GUARD_END(ctx)
}

strata_status strata_tsv_load(strata_ctx* ctx, const char* text, uint64_t text_len, uint32_t arity, int trop,
                              const char* dict_bytes, const uint64_t* dict_off, uint64_t n_dict, uint32_t** out_cols,
                              int64_t** out_w, uint64_t* out_rows, char** new_bytes, uint64_t** new_off,
                              uint64_t* n_new, uint64_t* err_line, uint32_t* err_col) {
  if (!ctx) return STRATA_E_INVALID;
  if (arity < 1 || arity > 2) return bad(ctx, "arity must be 1 or 2");
  if ((text_len && !text) || (n_dict && (!dict_bytes || !dict_off)) || !out_cols || !out_rows || !new_bytes ||
      !new_off || !n_new || (trop && !out_w))
    return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  if (err_line) *err_line = 0;
  if (err_col) *err_col = 0;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  sk::TsvResult r = sk::tsv_load(ctx, text, text_len, arity, trop != 0, dict_bytes, dict_off, n_dict);
  if (r.err_kind) {
    if (err_line) *err_line = r.err_line;
    if (err_col) *err_col = r.err_col;
    const std::string at = "line " + std::to_string(r.err_line) + ": ";
    if (r.err_kind == 1) return bad(ctx, (at + "expects " + std::to_string(arity + (trop ? 1 : 0)) + " column(s)").c_str());
    if (r.err_kind == 2) return bad(ctx, (at + "empty value in column " + std::to_string(r.err_col)).c_str());
    return bad(ctx, (at + "needs a trailing integer weight").c_str());
  }
  *out_cols = r.cols;
  if (out_w) *out_w = r.w;
  else std::free(r.w);
  *out_rows = r.rows;
  *new_bytes = r.new_bytes;
  *new_off = r.new_off;
  *n_new = r.n_new;
  SK_GUARD_END(ctx)
}

strata_status strata_rel_render(strata_ctx* ctx, const strata_rel* rel, const char* name, const char* dict_bytes,
                                const uint64_t* dict_off, uint64_t n_dict, char** out_text, uint64_t* out_len) {
  if (!ctx || !rel || !name || !out_text || !out_len || (n_dict && (!dict_bytes || !dict_off)))
    return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  static const uint64_t zero = 0;
  *out_len = sk::render_rel(ctx, rel, name, dict_bytes, n_dict ? dict_off : &zero, n_dict, out_text);
  SK_GUARD_END(ctx)
}

strata_status strata_op_select(strata_ctx* ctx, int key_bytes, const void* d_in, const int64_t* d_w, uint64_t n,
                               int shift, int mode, uint64_t value, void* d_out, int64_t* d_out_w, uint64_t* out_n) {
  if (!ctx) return STRATA_E_INVALID;
  if (key_bytes != 4 && key_bytes != 8) return bad(ctx, "key_bytes must be 4 or 8");
  if (mode < 0 || mode > 2) return bad(ctx, "mode must be 0 (c0 == c1), 1 (c0 == value) or 2 (c1 == value)");
  if (shift < 0 || shift > 8 * key_bytes) return bad(ctx, "shift outside [0, key bits]");
  if (!out_n || (n && (!d_in || !d_out || (d_w && !d_out_w)))) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  if (key_bytes == 4)
    *out_n = sk::op_select<uint32_t>(ctx, (const uint32_t*)d_in, d_w, n, shift, mode, value, (uint32_t*)d_out, d_out_w);
  else
    *out_n = sk::op_select<uint64_t>(ctx, (const uint64_t*)d_in, d_w, n, shift, mode, value, (uint64_t*)d_out, d_out_w);
  SK_GUARD_END(ctx)
}

strata_status strata_op_intersect(strata_ctx* ctx, int key_bytes, const void* d_a, const int64_t* d_aw, uint64_t na,
                                  const void* d_b, const int64_t* d_bw, uint64_t nb, void* d_out, int64_t* d_out_w,
                                  uint64_t* out_n) {
  if (!ctx) return STRATA_E_INVALID;
  if (key_bytes != 4 && key_bytes != 8) return bad(ctx, "key_bytes must be 4 or 8");
  if ((d_aw == nullptr) != (d_bw == nullptr)) return bad(ctx, "weights for both inputs or for neither");
  if (!out_n || (na && (!d_a || !d_out || (d_aw && !d_out_w))) || (nb && !d_b)) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  if (key_bytes == 4)
    *out_n = sk::op_intersect<uint32_t>(ctx, (const uint32_t*)d_a, d_aw, na, (const uint32_t*)d_b, d_bw, nb,
                                        (uint32_t*)d_out, d_out_w);
  else
    *out_n = sk::op_intersect<uint64_t>(ctx, (const uint64_t*)d_a, d_aw, na, (const uint64_t*)d_b, d_bw, nb,
                                        (uint64_t*)d_out, d_out_w);
  SK_GUARD_END(ctx)
}

strata_status strata_op_semijoin(strata_ctx* ctx, int key_bytes, const void* d_rows, const int64_t* d_w, uint64_t n,
                                 const void* d_probe, const void* d_b, uint64_t nb, int anti, void* d_out,
                                 int64_t* d_out_w, uint64_t* out_n) {
  if (!ctx) return STRATA_E_INVALID;
  if (key_bytes != 4 && key_bytes != 8) return bad(ctx, "key_bytes must be 4 or 8");
  if (!out_n || (n && (!d_rows || !d_out || (d_w && !d_out_w))) || (nb && !d_b)) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  if (key_bytes == 4)
    *out_n = sk::op_semijoin<uint32_t>(ctx, (const uint32_t*)d_rows, d_w, n, (const uint32_t*)d_probe,
                                       (const uint32_t*)d_b, nb, anti != 0, (uint32_t*)d_out, d_out_w);
  else
    *out_n = sk::op_semijoin<uint64_t>(ctx, (const uint64_t*)d_rows, d_w, n, (const uint64_t*)d_probe,
                                       (const uint64_t*)d_b, nb, anti != 0, (uint64_t*)d_out, d_out_w);
  SK_GUARD_END(ctx)
}

strata_status strata_op_join(strata_ctx* ctx, int key_bytes, const void* d_a, const int64_t* d_aw, uint64_t na,
                             int a_shift, const void* d_b, const int64_t* d_bw, uint64_t nb, int b_shift, int out_shift,
                             void* d_out, int64_t* d_out_w, uint64_t out_cap, uint64_t* out_n) {
  if (!ctx) return STRATA_E_INVALID;
  if (key_bytes != 4 && key_bytes != 8) return bad(ctx, "key_bytes must be 4 or 8");
  const int kbits = 8 * key_bytes;
  if (a_shift < 1 || a_shift >= kbits || b_shift < 1 || b_shift >= kbits || out_shift < 1 || out_shift >= kbits)
    return bad(ctx, "column shifts must lie in [1, key bits)");
  if (!out_n || (na && !d_a) || (nb && !d_b)) return bad(ctx, "NULL argument");
  if ((d_aw == nullptr) != (d_bw == nullptr)) return bad(ctx, "weights for both inputs or for neither");
  if (d_out && d_aw && !d_out_w) return bad(ctx, "Trop join needs an output weight column");
  if (na > sk::kMaxSortN || nb > sk::kMaxSortN) return bad(ctx, "n is limited to 2^30 - 1 per call");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  bool written = false;
  uint64_t t;
  if (key_bytes == 4)
    t = sk::op_join<uint32_t>(ctx, (const uint32_t*)d_a, d_aw, na, a_shift, (const uint32_t*)d_b, d_bw, nb, b_shift,
                              out_shift, (uint32_t*)d_out, d_out_w, out_cap, &written);
  else
    t = sk::op_join<uint64_t>(ctx, (const uint64_t*)d_a, d_aw, na, a_shift, (const uint64_t*)d_b, d_bw, nb, b_shift,
                              out_shift, (uint64_t*)d_out, d_out_w, out_cap, &written);
  *out_n = t;
  if (d_out && !written) return bad(ctx, "output capacity below the binding count (returned in *out_n)");
  SK_GUARD_END(ctx)
}

strata_status strata_op_project(strata_ctx* ctx, int key_bytes_in, const void* d_in, uint64_t n, int in_shift,
                                int sel_hi, int sel_lo, uint64_t const_hi, uint64_t const_lo, int key_bytes_out,
                                int out_shift, void* d_out) {
  if (!ctx) return STRATA_E_INVALID;
  if ((key_bytes_in != 4 && key_bytes_in != 8) || (key_bytes_out != 4 && key_bytes_out != 8))
    return bad(ctx, "key bytes must be 4 or 8");
  if (sel_lo < 0 || sel_lo > 2 || sel_hi < 0 || sel_hi > 3) return bad(ctx, "column selectors: 0 c0, 1 c1, 2 constant (3: none, hi only)");
  if (in_shift < 0 || in_shift > 8 * key_bytes_in) return bad(ctx, "in_shift outside [0, key bits]");
  if (sel_hi != 3 && (out_shift < 1 || out_shift >= 8 * key_bytes_out)) return bad(ctx, "out_shift outside [1, key bits)");
  if (n && (!d_in || !d_out)) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  if (key_bytes_in == 4 && key_bytes_out == 4)
    sk::op_project<uint32_t, uint32_t>(ctx, (const uint32_t*)d_in, n, in_shift, sel_hi, sel_lo, const_hi, const_lo,
                                       out_shift, (uint32_t*)d_out);
  else if (key_bytes_in == 4)
    sk::op_project<uint32_t, uint64_t>(ctx, (const uint32_t*)d_in, n, in_shift, sel_hi, sel_lo, const_hi, const_lo,
                                       out_shift, (uint64_t*)d_out);
  else if (key_bytes_out == 4)
    sk::op_project<uint64_t, uint32_t>(ctx, (const uint64_t*)d_in, n, in_shift, sel_hi, sel_lo, const_hi, const_lo,
                                       out_shift, (uint32_t*)d_out);
  else
    sk::op_project<uint64_t, uint64_t>(ctx, (const uint64_t*)d_in, n, in_shift, sel_hi, sel_lo, const_hi, const_lo,
                                       out_shift, (uint64_t*)d_out);
  SK_GUARD_END(ctx)
}

strata_status strata_op_aggregate(strata_ctx* ctx, int key_bytes, const void* d_keys, const int64_t* d_vals,
                                  uint64_t n, int group_shift, int op, void* d_groups, int64_t* d_out, uint64_t* out_n) {
  if (!ctx) return STRATA_E_INVALID;
  if (key_bytes != 4 && key_bytes != 8) return bad(ctx, "key_bytes must be 4 or 8");
  if (op < 0 || op > 3) return bad(ctx, "op must be 0 count, 1 sum, 2 min or 3 max");
  if (group_shift < 0 || group_shift > 8 * key_bytes) return bad(ctx, "group_shift outside [0, key bits]");
  if (!out_n || (n && (!d_keys || !d_groups || !d_out || (op && !d_vals)))) return bad(ctx, "NULL argument");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  if (key_bytes == 4)
    *out_n = sk::op_aggregate<uint32_t>(ctx, (const uint32_t*)d_keys, d_vals, n, group_shift, op, (uint32_t*)d_groups,
                                        d_out);
  else
    *out_n = sk::op_aggregate<uint64_t>(ctx, (const uint64_t*)d_keys, d_vals, n, group_shift, op, (uint64_t*)d_groups,
                                        d_out);
  SK_GUARD_END(ctx)
}

strata_status strata_op_merge(strata_ctx* ctx, int key_bytes, const void* d_a, const int64_t* d_aw, uint64_t na,
                              const void* d_b, const int64_t* d_bw, uint64_t nb, void* d_out, int64_t* d_out_w) {
  if (!ctx) return STRATA_E_INVALID;
  if (key_bytes != 4 && key_bytes != 8) return bad(ctx, "key_bytes must be 4 or 8");
  const bool trop = d_aw || d_bw || d_out_w;
  if ((na && !d_a) || (nb && !d_b) || ((na || nb) && !d_out)) return bad(ctx, "NULL argument");
  if (trop && ((na && !d_aw) || (nb && !d_bw) || !d_out_w)) return bad(ctx, "weights must be given for all or none");
  if (set_device(ctx) != STRATA_OK) return STRATA_E_CUDA;
  SK_GUARD_BEGIN
  sk::reset_status(ctx);
  if (key_bytes == 4) {
    if (trop) sk::merge_disjoint<uint32_t, int64_t, true>(ctx, (const uint32_t*)d_a, d_aw, na, (const uint32_t*)d_b, d_bw, nb, (uint32_t*)d_out, d_out_w);
    else sk::merge_disjoint<uint32_t, int32_t, false>(ctx, (const uint32_t*)d_a, nullptr, na, (const uint32_t*)d_b, nullptr, nb, (uint32_t*)d_out, nullptr);
  } else {
    if (trop) sk::merge_disjoint<uint64_t, int64_t, true>(ctx, (const uint64_t*)d_a, d_aw, na, (const uint64_t*)d_b, d_bw, nb, (uint64_t*)d_out, d_out_w);
    else sk::merge_disjoint<uint64_t, int32_t, false>(ctx, (const uint64_t*)d_a, nullptr, na, (const uint64_t*)d_b, nullptr, nb, (uint64_t*)d_out, nullptr);
  }
  sk::sync_and_check(ctx);
  SK_GUARD_END(ctx)
}

}  // extern "C"
