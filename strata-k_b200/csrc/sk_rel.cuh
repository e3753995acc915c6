// sk_rel.cuh — the device-resident relation handle and the driver interface
// shared by the fixpoint drivers, the WCOJ kernels and the C ABI.
#pragma once

#include "sk_common.cuh"

// A sorted, deduplicated binary relation held on the device.
// key = (c0 << shift) | c1 in a 4- or 8-byte word; Trop weights are int32
// (narrow) or int64 (wide) with +inf encoded as the type's maximum.
struct strata_rel {
  bool trop = false;
  int key_bytes = 4;
  int w_bytes = 0;
  int shift = 0;
  uint64_t n = 0;
  void* keys = nullptr;
  void* w = nullptr;
};

namespace sk {

// Device columns of an input relation (weights / inf mask optional).
struct EdgeCols {
  const uint32_t* src = nullptr;
  const uint32_t* dst = nullptr;
  const int64_t* w = nullptr;
  const uint8_t* inf = nullptr;
  uint64_t n = 0;
};

strata_rel* fix_tc_bool(strata_ctx* ctx, const EdgeCols& e, strata_fix_stats* st);
strata_rel* fix_trop_paths(strata_ctx* ctx, const EdgeCols& e, strata_fix_stats* st);
strata_rel* fix_mssp(strata_ctx* ctx, const uint32_t* sources, const int64_t* src_w,
                     const uint8_t* src_inf, uint64_t n_sources, const EdgeCols& e,
                     strata_fix_stats* st);

uint64_t count_triangle_pattern(strata_ctx* ctx, const uint32_t* x, const uint32_t* y, uint64_t n);

void tc_bool_batch(strata_ctx* ctx, uint32_t n_inst, const uint32_t* nodes, const uint64_t* edge_off,
                   const uint32_t* d_src, const uint32_t* d_dst, int mode, uint64_t* counts, uint64_t* fps,
                   uint32_t* rounds, strata_batch_stats* st);
bool tc_bool_bitset_fits(strata_ctx* ctx, uint64_t n_src, uint64_t n_dst, uint64_t m);
template <class K>
uint64_t tc_bool_bitset(strata_ctx* ctx, const uint32_t* d_src, const uint32_t* d_dst, uint64_t m, uint64_t n_src,
                        uint64_t n_dst, int b1, DBuf<K>& out, uint64_t* rounds, uint64_t* round_bytes);
uint64_t count_triangles_undirected(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n);
uint64_t count_4cliques_undirected(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n);
uint64_t binary_plan_intermediate(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n);
uint64_t intern_terms(strata_ctx* ctx, const uint64_t* keys, uint64_t n, uint32_t* ids);

void rel_to_host(strata_ctx* ctx, const strata_rel* rel, uint32_t* src, uint32_t* dst, int64_t* w,
                 uint8_t* inf);
uint64_t rel_fingerprint(strata_ctx* ctx, const strata_rel* rel);
void rel_free(strata_ctx* ctx, strata_rel* rel);

}  // namespace sk
