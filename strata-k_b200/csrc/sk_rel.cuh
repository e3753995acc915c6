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
  int64_t wshift = 0;  // Trop: finite value = weight code + wshift
  uint64_t n = 0;
  void* keys = nullptr;
  void* w = nullptr;
};

// Compiled provenance circuits of a set of queries, levelled per query
// (sk_circuit.cu).
struct strata_circuits {
  uint32_t n_queries = 0;
  uint32_t n_leaves = 0;
  uint64_t n_nodes = 0;
  uint32_t max_levels = 0;
  // device arrays
  uint8_t* kind = nullptr;      // 0 leaf, 1 neg leaf, 2 and, 3 or, 4 true, 5 false
  uint32_t* a = nullptr;        // leaf index, or first child (index into `ch`)
  uint32_t* b = nullptr;        // child count
  uint32_t* ch = nullptr;       // children (global node indices)
  uint64_t* qnode = nullptr;    // first node of query q (n_queries + 1)
  uint32_t* root = nullptr;     // root node of query q (global index)
  uint64_t* qlevel = nullptr;   // first level of query q in `lvl` (n_queries + 1)
  uint32_t* lvl = nullptr;      // level boundaries: node offsets relative to qnode[q]
  float* val = nullptr;         // forward values: high parts of the float-float pairs
  float* val_lo = nullptr;      // forward values: low parts (value = val + val_lo)
  float* adj = nullptr;         // adjoints
  uint64_t n_children = 0;
};

// One rank's share of a sharded bit-row closure (sk_bitset.cu): path rows
// [lo, hi) of n nodes (per = ceil(n / world) rows per rank), the rows'
// out-edge CSR with global neighbour ids, and the rank's path bit rows.
struct strata_tc_shard {
  strata_ctx* ctx = nullptr;
  uint32_t n = 0, rank = 0, world = 0, per = 0, lo = 0, hi = 0, w4 = 0;
  uint64_t n_edges = 0, m = 0;
  // The caller's edge columns (device): valid only until the seed, which
  // copies what the rounds need and clears these.
  const uint32_t* src = nullptr;
  const uint32_t* dst = nullptr;
  bool seeded = false;  // F, nbr and the Δ slice hold data only after the seed
  sk::DBuf<uint64_t> off;
  sk::DBuf<uint32_t> nbr;
  sk::DBuf<uint4> F;
  sk::DBuf<unsigned long long> acc;  // counters: Δ' size, summary, bad-edge flag
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
uint64_t count_triangle_pattern_range(strata_ctx* ctx, const uint32_t* x, const uint32_t* y, uint64_t n,
                                      uint64_t u_lo, uint64_t u_hi);

void tc_bool_batch(strata_ctx* ctx, uint32_t n_inst, const uint32_t* nodes, const uint64_t* edge_off,
                   const uint32_t* d_src, const uint32_t* d_dst, int mode, uint64_t* counts, uint64_t* fps,
                   uint32_t* rounds, strata_batch_stats* st);
bool tc_bool_bitset_fits(strata_ctx* ctx, uint64_t n_src, uint64_t n_dst, uint64_t m);

void prov_tc_capture(strata_ctx* ctx, uint32_t n, const uint32_t* d_src, const uint32_t* d_dst, uint64_t m,
                     const double* d_prob, uint32_t k, uint32_t nq, const uint32_t* qs, const uint32_t* qt,
                     std::vector<std::vector<std::vector<uint32_t>>>& out, std::vector<uint32_t>& rounds_out,
                     strata_prov_stats* st);
strata_circuits* circuits_compile(strata_ctx* ctx, uint32_t nq, const uint64_t* proof_off, const uint64_t* lit_off,
                                  const int64_t* lits, uint32_t n_leaves, uint64_t max_nodes);
void circuits_free(strata_ctx* ctx, strata_circuits* c);
struct CircuitParts;
CircuitParts* circuit_parts_compile(uint32_t nq, const uint64_t* proof_off, const uint64_t* lit_off,
                                    const int64_t* lits, uint32_t n_leaves, uint64_t max_nodes);
void circuit_parts_free(CircuitParts* p);
uint64_t circuit_parts_nodes(const CircuitParts* p, uint32_t* max_levels);
uint32_t circuit_parts_queries(const CircuitParts* p);
void circuit_parts_eval64(const CircuitParts* p, const double* prob, double* out);
strata_circuits* circuit_parts_upload(strata_ctx* ctx, uint32_t n_parts, CircuitParts* const* parts,
                                      uint32_t n_leaves);
void circuits_forward(strata_ctx* ctx, const strata_circuits* c, const float* d_p, float* out32, double* out64);
void circuits_adjoint(strata_ctx* ctx, const strata_circuits* c, const float* d_p, const float* seed, double* grad,
                      int per_query, float* grad32);
template <class K>
uint64_t tc_bool_bitset(strata_ctx* ctx, const uint32_t* d_src, const uint32_t* d_dst, uint64_t m, uint64_t n_src,
                        uint64_t n_dst, int b1, DBuf<K>& out, uint64_t* rounds, uint64_t* round_bytes);
uint64_t count_triangles_undirected(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n);
uint64_t count_4cliques_undirected(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n);
uint64_t binary_plan_intermediate(strata_ctx* ctx, const uint32_t* a, const uint32_t* b, uint64_t n);
uint64_t intern_terms(strata_ctx* ctx, const uint64_t* keys, uint64_t n, uint32_t* ids);

void tc_shard_init(strata_ctx* ctx, strata_tc_shard* sh, uint32_t n, const uint32_t* d_src, const uint32_t* d_dst,
                   uint64_t m, uint32_t rank, uint32_t world);
uint64_t tc_shard_seed(strata_ctx* ctx, strata_tc_shard* sh, uint4* Dmine, uint8_t* fmine);
uint64_t tc_shard_round(strata_ctx* ctx, strata_tc_shard* sh, const uint4* Dfull, const uint8_t* ffull, uint4* Dmine,
                        uint8_t* fmine);
void tc_shard_summary(strata_ctx* ctx, strata_tc_shard* sh, uint64_t* count, uint64_t* fp);
uint64_t tc_shard_pack(strata_ctx* ctx, strata_tc_shard* sh, const uint4* Dmine, int64_t* out, uint64_t cap);
void tc_shard_unpack(strata_ctx* ctx, strata_tc_shard* sh, const int64_t* in, uint64_t n, uint4* Dfull,
                     uint8_t* ffull);

void rel_to_host(strata_ctx* ctx, const strata_rel* rel, uint32_t* src, uint32_t* dst, int64_t* w,
                 uint8_t* inf);
uint64_t rel_fingerprint(strata_ctx* ctx, const strata_rel* rel);
void rel_free(strata_ctx* ctx, strata_rel* rel);

}  // namespace sk
