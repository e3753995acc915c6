/*
 * strata_b200.h — C ABI of the B200 relational fixpoint engine.
 *
 * This is the drop-in boundary for the semi-naive fixpoint hot path of
 * Strata/K.  Every entry point takes plain pointers and sizes; nothing here
 * names a torch or Rust type.  A Rust crate binds it with `extern "C"`, Python
 * with ctypes (see the `strata_b200` package).
 *
 * Conventions (shared by every call):
 *   - Node / symbol ids are u32 (`SymbolId`, strata-ir/src/dict.rs:19).
 *   - A binary relation crosses the boundary column-wise: `src[i], dst[i]`.
 *   - A Trop weight crosses as `int64_t w[i]` plus an optional byte mask
 *     `inf[i]` (1 = +inf, 0 = Finite(w[i])).  A NULL mask means all finite.
 *     +inf is therefore distinct from every finite i64, matching
 *     `Weight::{Finite(i64), PosInf}` (strata-ir/src/trop.rs:35-40).
 *   - Inputs need not be sorted or deduplicated.  Outputs are sorted by
 *     `(src, dst)` ascending, deduplicated (Bool) or min-merged (Trop), which
 *     is `BTreeMap` order over `GroundVal::Sym` ids (strata-eval/src/store.rs:19).
 *   - Results whose size is unknown in advance are returned in buffers the
 *     library allocates with malloc; release them with `strata_free`.
 *   - Every call runs on the context's stream and returns when its result is
 *     complete.  A context must not be used by two threads at once; separate
 *     contexts are independent (no process-global state).
 *   - Finite(i64::MAX) is a legal weight.  STRATA_E_WEIGHT_RANGE is returned
 *     only when the finite weights span nearly all of i64 (sums within the
 *     round cap could reach both i64::MIN and i64::MAX), where no 64-bit
 *     code keeps every value apart from +inf.
 *   - Errors are `strata_status` codes; `strata_last_error(ctx)` gives the
 *     message.  The codes map 1:1 onto the reference's error variants:
 *       STRATA_E_OVERFLOW   <- EvalError::Overflow      (strata-eval/src/naive.rs:31)
 *       STRATA_E_NEG_CYCLE  <- EvalError::NegativeWeightCycle (naive.rs:45)
 *       STRATA_E_CUDA       <- GpuError::Cuda           (strata-gpu/src/lib.rs:18)
 *       STRATA_E_NOT_BUILT  <- GpuError::NotBuilt       (strata-gpu/src/lib.rs:16)
 */
#ifndef STRATA_B200_H
#define STRATA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum strata_status {
  STRATA_OK = 0,
  STRATA_E_INVALID = 1,      /* bad argument (NULL pointer, size limit, bad id) */
  STRATA_E_OOM = 2,          /* device allocation failed or context cap reached */
  STRATA_E_CUDA = 3,         /* CUDA runtime error */
  STRATA_E_OVERFLOW = 4,     /* Trop finite (x) overflowed i64 (checked add) */
  STRATA_E_NEG_CYCLE = 5,    /* Trop stratum exceeded the Bellman-Ford round cap */
  STRATA_E_TIMEOUT = 6,      /* a bounded device wait gave up (never a hang) */
  STRATA_E_UNSUPPORTED = 7,  /* rule shape / size outside what the engine runs */
  STRATA_E_NOT_BUILT = 8,    /* no CUDA device visible to this library */
  STRATA_E_WEIGHT_RANGE = 9  /* finite weights spanning nearly all of i64: no
                                64-bit code separates them from +inf */
} strata_status;

typedef struct strata_ctx strata_ctx;

/* Per-fixpoint statistics filled by the drivers (all optional: pass NULL). */
typedef struct strata_fix_stats {
  uint64_t rounds;          /* semi-naive delta rounds executed (bootstrap excluded) */
  uint64_t candidates;      /* join outputs summed over rounds */
  uint64_t result_tuples;   /* |final IDB relation| */
  uint64_t universe;        /* distinct ids in the EDB (Bellman-Ford cap basis) */
  uint32_t key_bits;        /* significant bits of a packed tuple key */
  uint32_t weight_bytes;    /* 0 (Bool), 4 (narrow Trop) or 8 (wide Trop) */
  double   device_ms;       /* device time of the fixpoint (CUDA events) */
  double   sort_ms, join_ms, diff_ms, merge_ms; /* per-phase device time */
  uint64_t sort_bytes, join_bytes, diff_bytes, merge_bytes; /* algorithmic bytes */
  uint32_t sort_launches, join_launches, diff_launches, merge_launches;
  uint32_t other_launches;
  uint32_t plan;            /* 1 sort-merge, 2 direct-addressed (see strata_ctx_set_plan) */
  double   setup_ms;        /* EDB indexing before the first round (profiling on) */
  double   finish_ms;       /* building the output relation after the last round (profiling on) */
} strata_fix_stats;

/* ---- context ------------------------------------------------------------ */

/* Create a context on CUDA device `device`.  `mem_cap_bytes` bounds the bytes
 * this context may hold on the device at once (0 = no cap).  Allocations past
 * the cap fail with STRATA_E_OOM instead of reaching the driver. */
strata_status strata_ctx_create(int device, uint64_t mem_cap_bytes, strata_ctx** out);
void strata_ctx_destroy(strata_ctx* ctx);
/* Use an existing cudaStream_t (passed as void*) for all work; NULL = own stream. */
strata_status strata_ctx_set_stream(strata_ctx* ctx, void* stream);
/* Wait for all work queued on the context's stream (the asynchronous calls). */
strata_status strata_ctx_synchronize(strata_ctx* ctx);
const char* strata_last_error(const strata_ctx* ctx);
/* Device bytes currently held and the high-water mark. */
strata_status strata_ctx_mem(const strata_ctx* ctx, uint64_t* in_use, uint64_t* peak);
/* Physical plan of the fixpoint rounds: 0 = automatic (direct-addressed when
 * the two column domains multiply to a small enough index and the weights
 * fit int32, else sort-merge), 1 = sort-merge (radix sort + run reduction +
 * merge-path diff every round), 2 = direct-addressed (a bitmap / int32 index
 * over (c0, c1); STRATA_E_UNSUPPORTED when it does not apply), 3 = bit rows
 * (Bool transitive closure only: path and Δ as bit rows over the Z domain,
 * one 128-bit OR joins 128 tuples; STRATA_E_UNSUPPORTED for other programs
 * or when the three bit matrices exceed 8 GB).  Automatic planning picks bit
 * rows for Bool closure when they fit.  Results are identical; only speed
 * and memory differ. */
strata_status strata_ctx_set_plan(strata_ctx* ctx, int plan);
/* Tuning knobs (speed only; results are identical for every value):
 *   STRATA_KNOB_SORT_ITEMS_U32  keys per thread of a radix tile, u32 keys: 11, 15, 19, 23
 *   STRATA_KNOB_SORT_ITEMS_U64  keys per thread of a radix tile, u64 keys: 7, 9, 13
 *   STRATA_KNOB_TRI_PROBE       triangle membership test: 1 shared-memory hash set,
 *                               2 binary search of the sorted out-list, 3 shared-memory
 *                               bitmap filter with queued binary searches
 *   STRATA_KNOB_BATCH_GRAPH_ROUNDS  bit-row rounds per CUDA-graph replay: 2, 4, 8, 16, 32
 *   STRATA_KNOB_BATCH_BLOCKS_PER_SM resident blocks per SM of the round kernel: 1..32
 *   STRATA_KNOB_BATCH_BUDGET_MB     cap on one batch wave's device bytes, in MiB (>= 1)
 *   STRATA_KNOB_SORT_RANK           radix digit ranking: 1 per-bit warp ballots, 2 match instruction,
 *                                   3 shared-memory peer masks
 *   STRATA_KNOB_DENSE_WORD_MEMBERS  direct-addressed rounds: Δ words with at least this many
 *                                   members take the bit-lane expand path: 1..33 (33 = never)
 *   STRATA_KNOB_WEIGHT_LANES        Trop weight lanes: 8 = always int64 (otherwise int32 lanes
 *                                   are used when every sum within the round cap provably fits)
 * value 0 restores the default (15 / 9 / 3 / 8 / occupancy limit / 70% of
 * reusable memory / shared masks / 24 / automatic).  Other values: STRATA_E_INVALID.
 * The autotuner (strata_b200.tune) sweeps these and caches the best per GPU.
 * No counterpart in the reference (its sort has no tile parameters). */
#define STRATA_KNOB_SORT_ITEMS_U32 1
#define STRATA_KNOB_SORT_ITEMS_U64 2
#define STRATA_KNOB_TRI_PROBE 3
#define STRATA_KNOB_BATCH_GRAPH_ROUNDS 4
#define STRATA_KNOB_BATCH_BLOCKS_PER_SM 5
#define STRATA_KNOB_BATCH_BUDGET_MB 6
#define STRATA_KNOB_SORT_RANK 7
#define STRATA_KNOB_DENSE_WORD_MEMBERS 8
#define STRATA_KNOB_WEIGHT_LANES 9
strata_status strata_ctx_set_knob(strata_ctx* ctx, int knob, int value);
/* Enable per-phase CUDA-event timing in strata_fix_stats (adds event records). */
strata_status strata_ctx_set_profiling(strata_ctx* ctx, int enabled);
/* Number of kernels this context launched so far (monotone counter). */
uint64_t strata_ctx_launches(const strata_ctx* ctx);
/* Per-kernel accounting collected while profiling is on: launches, summed
 * CUDA-event duration and algorithmic bytes moved.  Kernel ids:
 * 0 radix pass, 1 expand emit, 2 expand offsets, 3 run reduction,
 * 4 merge/diff, 5 radix histogram, 6 triangle count, 7 direct-addressed expand,
 * 8 bit-row round, 9 Prov_k round, 10 circuit pass, 11 sharded bit-row round. */
strata_status strata_ctx_kernel_stats(strata_ctx* ctx, int kernel, uint64_t* launches,
                                      double* ms, uint64_t* bytes);
strata_status strata_ctx_reset_kernel_stats(strata_ctx* ctx);
/* Release memory returned by the library. */
void strata_free(void* p);
const char* strata_version(void);

/* ---- whole-fixpoint drivers (host buffers) ------------------------------
 * These mirror strata-gpu's public functions (strata-gpu/src/lib.rs:67-147). */

/* Bool transitive closure: path(X,Y) :- edge(X,Y). path(X,Z) :- edge(X,Y), path(Y,Z).
 * Replaces `transitive_closure_bool(&[(u32,u32)])` (strata-gpu/src/lib.rs:67). */
strata_status strata_transitive_closure_bool(strata_ctx* ctx,
    const uint32_t* src, const uint32_t* dst, uint64_t n_edges,
    uint32_t** out_src, uint32_t** out_dst, uint64_t* out_n,
    strata_fix_stats* stats);

/* Trop all-pairs: reach(X,Y) :- edge(X,Y). reach(X,Z) :- edge(X,Y), reach(Y,Z).
 * Replaces `shortest_paths_trop(&[(u32,u32,i64)])` (strata-gpu/src/lib.rs:84).
 * The Bellman-Ford cap is the interpreter's: universe + 2 delta rounds
 * (strata-eval/src/seminaive.rs:96-103). */
strata_status strata_shortest_paths_trop(strata_ctx* ctx,
    const uint32_t* src, const uint32_t* dst, const int64_t* w, const uint8_t* inf,
    uint64_t n_edges,
    uint32_t** out_src, uint32_t** out_dst, int64_t** out_w, uint8_t** out_inf,
    uint64_t* out_n, strata_fix_stats* stats);

/* Trop multi-source: dist(S,Y) :- src(S), edge(S,Y). dist(S,Z) :- dist(S,Y), edge(Y,Z).
 * `sources[i]` with weight `src_w[i]` (NULL = the otimes identity Finite(0), how a
 * Bool fact enters Trop, strata-ir/src/trop.rs:44-45).  No reference GPU
 * counterpart; it replaces `run_semi_naive` (strata-eval/src/seminaive.rs:29)
 * for this rule shape. */
strata_status strata_mssp_trop(strata_ctx* ctx,
    const uint32_t* sources, const int64_t* src_w, const uint8_t* src_inf, uint64_t n_sources,
    const uint32_t* esrc, const uint32_t* edst, const int64_t* ew, const uint8_t* einf,
    uint64_t n_edges,
    uint32_t** out_src, uint32_t** out_dst, int64_t** out_w, uint8_t** out_inf,
    uint64_t* out_n, strata_fix_stats* stats);

/* Triangles of the undirected graph on the edges (self-loops and duplicates
 * ignored, both directions accepted).  Replaces `count_triangles`
 * (strata-gpu/src/lib.rs:99, strata-gpu/src/wcoj.rs:136). */
strata_status strata_count_triangles(strata_ctx* ctx,
    const uint32_t* a, const uint32_t* b, uint64_t n_edges, uint64_t* out_count);

/* 4-cliques of the undirected graph.  Replaces `count_4cliques`
 * (strata-gpu/src/lib.rs:114, strata-gpu/src/wcoj.rs:166). */
strata_status strata_count_4cliques(strata_ctx* ctx,
    const uint32_t* a, const uint32_t* b, uint64_t n_edges, uint64_t* out_count);

/* The count aggregate  n(count<X>) :- e(X,Y), e(Y,Z), e(X,Z)  over the directed
 * relation e exactly as given (deduplicated as a set, no orientation).  This is
 * `eval_aggregate_rule` + `fold_aggregate(Count)` for that body
 * (strata-eval/src/naive.rs:300-391). */
strata_status strata_count_triangle_pattern(strata_ctx* ctx,
    const uint32_t* x, const uint32_t* y, uint64_t n_edges, uint64_t* out_count);

/* Intern u64 term keys: ids[i] = rank of keys[i] among the distinct keys.
 * Replaces `intern_terms` (strata-gpu/src/lib.rs:133, sort.rs:206). */
strata_status strata_intern_terms(strata_ctx* ctx,
    const uint64_t* keys, uint64_t n, uint32_t* ids_out, uint64_t* n_distinct);

/* Σ_v d(v)^2 over the id-oriented simple graph: the binary-plan intermediate
 * WCOJ avoids.  Replaces `binary_plan_intermediate` (strata-gpu/src/lib.rs:140). */
strata_status strata_binary_plan_intermediate(strata_ctx* ctx,
    const uint32_t* a, const uint32_t* b, uint64_t n_edges, uint64_t* out);

/* ---- device-resident drivers ---------------------------------------------
 * Same fixpoints with inputs already in device memory (pointers from
 * cudaMalloc / torch).  The result stays on the device in a relation handle. */

typedef struct strata_rel strata_rel;

strata_status strata_tc_bool_dev(strata_ctx* ctx,
    const uint32_t* d_src, const uint32_t* d_dst, uint64_t n_edges,
    strata_rel** out, strata_fix_stats* stats);
strata_status strata_trop_paths_dev(strata_ctx* ctx,
    const uint32_t* d_src, const uint32_t* d_dst, const int64_t* d_w, const uint8_t* d_inf,
    uint64_t n_edges, strata_rel** out, strata_fix_stats* stats);
strata_status strata_mssp_trop_dev(strata_ctx* ctx,
    const uint32_t* d_sources, const int64_t* d_src_w, const uint8_t* d_src_inf, uint64_t n_sources,
    const uint32_t* d_esrc, const uint32_t* d_edst, const int64_t* d_ew, const uint8_t* d_einf,
    uint64_t n_edges, strata_rel** out, strata_fix_stats* stats);
strata_status strata_count_triangle_pattern_dev(strata_ctx* ctx,
    const uint32_t* d_x, const uint32_t* d_y, uint64_t n_edges, uint64_t* out_count);
/* The bindings with X in [x_lo, x_hi) only: the share of one rank when the
 * source vertices are split across GPUs (the edge list is replicated; the
 * shares add up to the full count). */
strata_status strata_count_triangle_pattern_range_dev(strata_ctx* ctx,
    const uint32_t* d_x, const uint32_t* d_y, uint64_t n_edges, uint64_t x_lo, uint64_t x_hi,
    uint64_t* out_count);

/* ---- batched Bool reachability ------------------------------------------
 * Many independent transitive closures in one call (the reference computes
 * one graph per `transitive_closure_bool` call, strata-gpu/src/lib.rs:67 and
 * tc.rs:31; this is its batched submission).  Instance i has nodes
 * [0, nodes[i]) and the edges src/dst[edge_off[i] .. edge_off[i+1]) (local
 * ids; duplicates allowed).  Each closure is summarised, not materialised:
 *   counts[i] = |path_i|,
 *   fps[i]    = Σ_{(X,Z) ∈ path_i} mix64(X) · c^Z  mod 2^64,
 *               mix64 = the splitmix64 finalizer, c = 0x9E3779B97F4A7C15,
 *   rounds[i] = semi-naive delta rounds (as strata_fix_stats.rounds).
 * mode 0: batched — instances are packed into memory-bounded waves and each
 *         semi-naive round of a wave is one persistent kernel over all of its
 *         active instances, replayed from a captured CUDA graph;
 * mode 1: one instance per launch — the same kernels, one instance at a time
 *         with host-driven rounds (the comparison baseline).
 * nodes / edge_off / outputs are host arrays; src / dst are device arrays
 * (`_dev`) or host arrays (plain form). */
typedef struct strata_batch_stats {
  uint64_t instances;
  uint64_t waves;           /* memory-bounded groups of instances */
  uint64_t graph_launches;  /* CUDA-graph replays (mode 0) */
  uint64_t round_launches;  /* round kernels launched (graph nodes included) */
  uint64_t rounds_max;      /* most rounds of any instance */
  uint64_t result_tuples;   /* Σ counts */
  uint64_t round_bytes;     /* algorithmic bytes of the rounds (profiling on) */
  uint64_t launches;        /* kernels launched by the call */
  double   device_ms;       /* CUDA-event time of the whole call */
} strata_batch_stats;

strata_status strata_tc_bool_batch_dev(strata_ctx* ctx, uint32_t n_inst, const uint32_t* nodes,
    const uint64_t* edge_off, const uint32_t* d_src, const uint32_t* d_dst, int mode,
    uint64_t* counts, uint64_t* fps, uint32_t* rounds, strata_batch_stats* stats);
strata_status strata_tc_bool_batch(strata_ctx* ctx, uint32_t n_inst, const uint32_t* nodes,
    const uint64_t* edge_off, const uint32_t* src, const uint32_t* dst, int mode,
    uint64_t* counts, uint64_t* fps, uint32_t* rounds, strata_batch_stats* stats);

/* ---- sharded Bool closure (one rank's share) -----------------------------
 * Rank `rank` of `world` owns the path rows X in [rank*P, min((rank+1)*P,
 * n_nodes)), P = ceil(n_nodes / world), as bit rows of `row_bytes` bytes
 * over the Z domain.  The only exchange is once per round: the caller
 * gathers every rank's Delta' slice (P rows, P row flags) into the full
 * Delta (world*P rows and flags, in rank order) that the next round reads
 * (an NCCL all-gather over NVLink), and sums the ranks' |Delta'|; the
 * closure is done when that sum is 0.  The rounds, the summed |path| and the
 * summed fingerprint sum mix64(X)*c^Z (mod 2^64, as strata_tc_bool_batch)
 * equal the single-device closure's.
 * Counterpart: the reference's sharding interface for joins
 * (strata-gpu/src/partition.rs:35-83, a CPU specification: tuples
 * hash-partitioned by join key, the whole join the union of the shard
 * joins); here path is partitioned by row and Delta replicated by the gather.
 * d_src / d_dst (m edges, device) must stay valid until the seed returns;
 * endpoints outside [0, n_nodes): STRATA_E_INVALID.  The share is seeded
 * exactly once: a second seed, or a round / summary before the seed, is
 * STRATA_E_INVALID. */
typedef struct strata_tc_shard strata_tc_shard;
strata_status strata_tc_shard_create(strata_ctx* ctx, uint32_t n_nodes, const uint32_t* d_src,
    const uint32_t* d_dst, uint64_t m, uint32_t rank, uint32_t world, strata_tc_shard** out);
strata_status strata_tc_shard_shape(const strata_tc_shard* sh, uint32_t* rows_per_rank, uint32_t* row_lo,
    uint32_t* row_hi, uint64_t* row_bytes);
/* Delta0 = path = the rank's edges: writes its Delta slice (P rows of
 * row_bytes, 16-byte aligned) and P row flags; *n_delta = |Delta0| of its rows. */
strata_status strata_tc_shard_seed(strata_ctx* ctx, strata_tc_shard* sh, void* d_delta_mine,
    uint8_t* d_flags_mine, uint64_t* n_delta);
/* One semi-naive round of the rank's rows from the gathered Delta and row
 * flags (neither may overlap the rank's output slice of the same kind:
 * STRATA_E_INVALID); *n_delta = |Delta'| of its rows. */
strata_status strata_tc_shard_round(strata_ctx* ctx, strata_tc_shard* sh, const void* d_delta_full,
    const uint8_t* d_flags_full, void* d_delta_mine, uint8_t* d_flags_mine, uint64_t* n_delta);
/* Sparse exchange of a round's Delta': the rank's nonzero 128-bit words as
 * (global word index, low 64 bits, high 64 bits) int64 triples.  pack writes
 * min(count, cap) triples to d_out (cap x 3 int64; slots past the count get
 * index -1) and *n_words = the count, so cap = 0 only counts.  unpack clears
 * the gathered Delta and row flags and scatters n triples (index -1 skipped)
 * into them; the triples may not overlap the gathered Delta.  Used instead of
 * the slice all-gather when the largest rank's count x 24 bytes is well below
 * the slice size. */
strata_status strata_tc_shard_pack(strata_ctx* ctx, strata_tc_shard* sh, const void* d_delta_mine,
    int64_t* d_out, uint64_t cap, uint64_t* n_words);
strata_status strata_tc_shard_unpack(strata_ctx* ctx, strata_tc_shard* sh, const int64_t* d_in, uint64_t n,
    void* d_delta_full, uint8_t* d_flags_full);
/* |path| of the rank's rows and their part of the fingerprint. */
strata_status strata_tc_shard_summary(strata_ctx* ctx, strata_tc_shard* sh, uint64_t* count,
    uint64_t* fingerprint);
/* Frees the share (its buffers return to the context's pool): call it before
 * strata_ctx_destroy of the context that created it. */
void strata_tc_shard_free(strata_tc_shard* sh);

/* ---- Prov_k capture and provenance circuits -----------------------------
 * The probabilistic reachability program
 *     path(X,Y) :- edge(X,Y).   path(X,Z) :- edge(X,Y), path(Y,Z).
 * with `path` Prov_k(k) (k <= 8) and every edge a probabilistic fact: edge i
 * (0-based, input order) is the leaf with literal i+1 and probability
 * d_prob[i].  Replaces `run_prov` (strata-eval/src/provenance.rs:217-283) +
 * `ProvDb::query` for this program, with the same naive-round semantics,
 * evaluated only for the targets of the query pairs (qs[q], qt[q]) (host
 * arrays).  Edge tuples must be distinct (STRATA_E_UNSUPPORTED otherwise);
 * proofs longer than 32 literals are refused (STRATA_E_UNSUPPORTED).
 * target_rounds (optional, one per distinct target in ascending order)
 * receives the rounds until that target's tuples stopped changing. */
typedef struct strata_prov_stats {
  uint64_t queries, targets, waves, rounds_max, max_proof_len, launches;
  double device_ms;
} strata_prov_stats;
typedef struct strata_proofs strata_proofs;
strata_status strata_prov_tc_capture(strata_ctx* ctx, uint32_t n_nodes, const uint32_t* d_src,
    const uint32_t* d_dst, uint64_t n_edges, const double* d_prob, uint32_t k, uint32_t n_queries,
    const uint32_t* qs, const uint32_t* qt, strata_proofs** out, uint32_t* target_rounds,
    strata_prov_stats* stats);
/* Sizes, then the flattened proof sets: query q owns proofs
 * [proof_off[q], proof_off[q+1]), proof p the literals [lit_off[p], lit_off[p+1])
 * (ascending; the proofs of a query in proof-set order). */
strata_status strata_proofs_shape(const strata_proofs* pr, uint32_t* n_queries, uint64_t* n_proofs,
    uint64_t* n_lits);
strata_status strata_proofs_export(const strata_proofs* pr, uint64_t* proof_off, uint64_t* lit_off,
    int64_t* lits);
void strata_proofs_free(strata_proofs* pr);

/* Exact compilation of each query's proof DNF (signed literals ±(leaf+1),
 * host arrays in the layout above) to a deterministic, decomposable circuit
 * by Shannon expansion (strata-prob/src/compile.rs:80-150), kept on the
 * device.  max_nodes bounds each query's circuit (0 = 2^20, the reference's
 * default); STRATA_E_UNSUPPORTED past it. */
typedef struct strata_circuits strata_circuits;
strata_status strata_circuits_compile(strata_ctx* ctx, uint32_t n_queries, const uint64_t* proof_off,
    const uint64_t* lit_off, const int64_t* lits, uint32_t n_leaves, uint64_t max_nodes,
    strata_circuits** out);
/* The same in two steps, so the host compilation of one group of queries
 * can run on another thread while the device captures the next group:
 * strata_circuits_compile_host touches no device and no context (thread-safe;
 * its error message is strata_circuit_parts_error() on the calling thread),
 * strata_circuits_upload concatenates parts (queries in part order). */
typedef struct strata_circuit_parts strata_circuit_parts;
strata_status strata_circuits_compile_host(uint32_t n_queries, const uint64_t* proof_off,
    const uint64_t* lit_off, const int64_t* lits, uint32_t n_leaves, uint64_t max_nodes,
    strata_circuit_parts** out);
const char* strata_circuit_parts_error(void);
strata_status strata_circuits_upload(strata_ctx* ctx, uint32_t n_parts, strata_circuit_parts* const* parts,
    uint32_t n_leaves, strata_circuits** out);
void strata_circuit_parts_free(strata_circuit_parts* parts);
/* Node count / levels of host-compiled parts, and their FP64 evaluation on
 * the host (P per query for FP64 leaf probabilities) — checks of the
 * compiler that need no device. */
strata_status strata_circuit_parts_shape(const strata_circuit_parts* parts, uint32_t* n_queries,
    uint64_t* n_nodes, uint32_t* max_levels);
strata_status strata_circuit_parts_eval64(const strata_circuit_parts* parts, const double* prob, double* out);
strata_status strata_circuits_shape(const strata_circuits* c, uint64_t* n_nodes, uint32_t* max_levels);
/* Weighted model counts (Circuit::wmc, circuit.rs:57-63) of every query for
 * leaf probabilities d_p (FP32, n_leaves): FP32 nodes, the root's sum in
 * FP64; d_out (FP32) and/or d_out64 (FP64) per query.  Asynchronous on the
 * context's stream; one circuit set must not be evaluated concurrently. */
strata_status strata_circuits_forward(strata_ctx* ctx, const strata_circuits* c, const float* d_p,
    float* d_out, double* d_out64);
/* Vector-Jacobian product: d_grad64[i] = Σ_q d_seed[q] · ∂P_q/∂p_i (FP32
 * adjoints, FP64 leaf sums; d_seed NULL = all ones); d_grad32 optional FP32
 * copy.  The torch.autograd backward of the forward above. */
strata_status strata_circuits_vjp(strata_ctx* ctx, const strata_circuits* c, const float* d_p,
    const float* d_seed, double* d_grad64, float* d_grad32);
/* Per-query gradients (Circuit::grad, circuit.rs:68-106): d_grads is
 * [n_queries][n_leaves] FP64 (the `?grad` rows). */
strata_status strata_circuits_grads(strata_ctx* ctx, const strata_circuits* c, const float* d_p,
    double* d_grads);
void strata_circuits_free(strata_ctx* ctx, strata_circuits* c);

/* ---- ASP grounding-simplify filter ----------------------------------------
 * Replaces `simplify_filter` (strata-gpu/src/asp.rs:121-136, semantics of
 * simplify_filter_cpu / keep_literal :53-100) for a ground
 * program in CSR form: rule i has head[i] (atom id, -1 for a constraint) and
 * the signed body literals body_lit[body_start[i] .. body_start[i+1]) (+(a+1)
 * positive, -(a+1) negative).  A rule whose positive atom is impossible
 * (poss[a] == 0) or whose negative atom is certain (cert[a] != 0) is dropped;
 * a surviving rule loses its certain positive and impossible negative
 * literals.  Returns malloc'd arrays (free with strata_free) in rule order;
 * a literal naming no atom (0 or beyond n_atoms) is STRATA_E_CUDA with a
 * bounds message and nothing is returned. */
strata_status strata_asp_simplify_filter(strata_ctx* ctx, uint64_t n_rules, const int32_t* head,
    const uint32_t* body_start, const int32_t* body_lit, uint64_t n_atoms, const uint8_t* poss, const uint8_t* cert,
    int32_t** out_head, uint32_t** out_body_start, int32_t** out_body_lit, uint64_t* out_n);

/* ---- input and output contracts on the device ----------------------------
 * One Soufflé TSV input file (strata-k/src/input.rs:53-197, 216-232): lines
 * split on '\n' with trailing '\r's dropped and empty lines skipped; each row
 * `arity` (1 or 2) tab-separated symbol cells, plus a trailing weight cell
 * parsed as `trim().parse::<i64>()` when `trop`.  Symbols are interned
 * first-seen (strata-ir/src/dict.rs:35-43) in row order, column order, after
 * the n_dict strings of the current dictionary (string i =
 * dict_bytes[dict_off[i] .. dict_off[i+1]), id i).  Returns malloc'd (free
 * with strata_free): out_cols (column-major: column c of row r at
 * c * out_rows + r), out_w (trop), and the new symbols in id order (ids n_dict
 * .. n_dict + n_new - 1: new_bytes[new_off[j] .. new_off[j+1]), n_new + 1
 * offsets).  A bad row returns STRATA_E_INVALID with *err_line = its 1-based
 * line (the first one) and *err_col the empty column (else 0); nothing is
 * returned and the dictionary is not extended.  The interning hashes are
 * verified byte by byte: ids are exact. */
strata_status strata_tsv_load(strata_ctx* ctx, const char* text, uint64_t text_len, uint32_t arity, int trop,
    const char* dict_bytes, const uint64_t* dict_off, uint64_t n_dict, uint32_t** out_cols, int64_t** out_w,
    uint64_t* out_rows, char** new_bytes, uint64_t** new_off, uint64_t* n_new, uint64_t* err_line,
    uint32_t* err_col);

/* The canonical text of a binary relation (render_db for one relation,
 * strata-cli/src/render.rs:29-54, 87-92): one line per tuple in id order,
 * `name(a, b)\n`, with ` = w` or ` = inf` for Trop; symbol names from the
 * dictionary (n_dict strings as above; an id it lacks prints `?`).  Built on
 * the device; *out_text is malloc'd and NUL-terminated (free with
 * strata_free), *out_len its length without the NUL. */
strata_status strata_rel_render(strata_ctx* ctx, const strata_rel* rel, const char* name, const char* dict_bytes,
    const uint64_t* dict_off, uint64_t n_dict, char** out_text, uint64_t* out_len);

/* Relation handle accessors. */
strata_status strata_rel_size(const strata_rel* rel, uint64_t* n);
strata_status strata_rel_is_trop(const strata_rel* rel, int* is_trop);
/* Copy out into caller buffers of strata_rel_size() entries; w / inf may be
 * NULL (ignored for Bool relations). */
strata_status strata_rel_to_host(strata_ctx* ctx, const strata_rel* rel,
    uint32_t* src, uint32_t* dst, int64_t* w, uint8_t* inf);
/* Order-independent 64-bit fingerprint of the relation's tuples (and
 * weights), for parity checks that must not copy the relation out. */
strata_status strata_rel_fingerprint(strata_ctx* ctx, const strata_rel* rel, uint64_t* fp);
void strata_rel_free(strata_ctx* ctx, strata_rel* rel);

/* ---- operator surface (device pointers) ----------------------------------
 * The interpreter's operators (strata-eval/src/seminaive.rs:114-298,
 * store.rs:34-48) on packed sorted key columns.  A packed key is
 * (c0 << shift) | c1 in a u32 (key_bytes = 4) or u64 (key_bytes = 8).
 * `n` is limited to 2^30 - 1 per call, except for strata_op_sort (2^32 - 1). */

/* Stable LSD radix sort of keys (and optional 4- or 8-byte values) on the low
 * `key_bits` bits.  Sorted output goes to keys_out / vals_out; the inputs are
 * left unchanged. */
strata_status strata_op_sort(strata_ctx* ctx, int key_bytes, int val_bytes,
    const void* d_keys_in, const void* d_vals_in, void* d_keys_out, void* d_vals_out,
    uint64_t n, int key_bits);

/* Bool dedup + difference (Δ = new \ full, seminaive.rs:192-209): from sorted
 * keys with duplicates, write the distinct keys absent from sorted unique
 * `full` to `out` (capacity n); *out_n receives the count.  full may be empty. */
strata_status strata_op_dedup_diff(strata_ctx* ctx, int key_bytes,
    const void* d_cand, uint64_t n, const void* d_full, uint64_t n_full,
    void* d_out, uint64_t* out_n);

/* Trop min-merge + improvement (Relation::combine, store.rs:34-48): from sorted
 * keys with int64 weights (INT64_MAX = +inf), reduce each key to its minimum;
 * keys new to `full` or strictly better than full's weight go to out_keys/out_w.
 * Strictly-better weights are also written into d_full_w in place. */
strata_status strata_op_min_improve(strata_ctx* ctx, int key_bytes,
    const void* d_cand, const int64_t* d_cand_w, uint64_t n,
    const void* d_full, int64_t* d_full_w, uint64_t n_full,
    void* d_out_keys, int64_t* d_out_w, uint64_t* out_n);

/* ⊕-combine a batch of derivations (Relation::combine, store.rs:34-48): from
 * sorted keys with duplicates, one row per key — Bool: the distinct keys;
 * Trop (d_w given): the minimum weight.  *out_n = distinct keys (capacity n).
 * The outputs may not overlap the inputs (STRATA_E_INVALID). */
strata_status strata_op_reduce(strata_ctx* ctx, int key_bytes, const void* d_keys, const int64_t* d_w, uint64_t n,
    void* d_out, int64_t* d_out_w, uint64_t* out_n);

/* Apply a round's reduced derivations to a relation and take the next Δ
 * (apply_round, seminaive.rs:183-208): full_out = full ⊕ cand (Bool union;
 * Trop min per key), delta = the keys of cand new to full (Trop: or strictly
 * below full's weight) with their merged values.  Both inputs sorted and
 * unique; capacities n_full + n_cand (full_out) and n_cand (delta); the
 * outputs may not overlap the inputs (STRATA_E_INVALID). */
strata_status strata_op_merge_diff(strata_ctx* ctx, int key_bytes, const void* d_full, const int64_t* d_full_w,
    uint64_t n_full, const void* d_cand, const int64_t* d_cand_w, uint64_t n_cand,
    void* d_full_out, int64_t* d_full_out_w, void* d_delta, int64_t* d_delta_w,
    uint64_t* out_full_n, uint64_t* out_delta_n);

/* Scan with unification (`unify`, strata-eval/src/naive.rs:407-455) for an
 * atom with a repeated variable or a constant: the rows of packed keys
 * (c0 << shift) | c1 with c0 == c1 (mode 0), c0 == value (mode 1) or
 * c1 == value (mode 2), in input order, weights carried (optional).
 * *out_n = rows kept (capacity n). */
strata_status strata_op_select(strata_ctx* ctx, int key_bytes, const void* d_in, const int64_t* d_w, uint64_t n,
    int shift, int mode, uint64_t value, void* d_out, int64_t* d_out_w, uint64_t* out_n);

/* Two atoms over the same variables, p(X,Y), q(X,Y) (`solve` binding both
 * columns): the keys of a (any order) that are in b (sorted ascending), in
 * a's order; with weights on both, the Trop product (INT64_MAX = +inf,
 * STRATA_E_OVERFLOW on a finite sum past i64).  *out_n = rows kept. */
strata_status strata_op_intersect(strata_ctx* ctx, int key_bytes, const void* d_a, const int64_t* d_aw, uint64_t na,
    const void* d_b, const int64_t* d_bw, uint64_t nb, void* d_out, int64_t* d_out_w, uint64_t* out_n);

/* Stratified negation (`negation_holds`, strata-eval/src/naive.rs:537-566):
 * keep row i of d_rows (weights carried) when probe[i] — the key of the
 * negated atom under row i's binding, from strata_op_project; NULL = the row
 * key itself — is absent from the sorted relation b (anti != 0), or present
 * (anti == 0, a semi-join).  In input order; *out_n = rows kept. */
strata_status strata_op_semijoin(strata_ctx* ctx, int key_bytes, const void* d_rows, const int64_t* d_w, uint64_t n,
    const void* d_probe, const void* d_b, uint64_t nb, int anti, void* d_out, int64_t* d_out_w, uint64_t* out_n);

/* One binary rule body  h(X,Z) :- a(X,Y), b(Y,Z)  (`solve` over two atoms,
 * strata-eval/src/seminaive.rs:215-298, with the head built as (X, Z),
 * `build_head` naive.rs:526).  a = (X << a_shift) | Y in any order (a Δ, or
 * a full relation); b = (Y << b_shift) | Z sorted ascending (strata_op_sort).
 * Every binding is written as (X << out_shift) | Z, in a's order, unsorted
 * and with duplicates; with weights (both d_aw and d_bw, int64, INT64_MAX =
 * +inf) the output weight is the Trop product (checked i64 add,
 * STRATA_E_OVERFLOW; Ann::otimes, value.rs:56).  *out_n receives the binding
 * count; pass d_out = NULL to size the output first.  out_cap below the
 * count is STRATA_E_INVALID (nothing written).  Shifts lie in [1, key bits);
 * the caller picks out_shift so the output keys fit.  Finite weights on this
 * surface are at most INT64_MAX - 2 (STRATA_E_WEIGHT_RANGE otherwise). */
strata_status strata_op_join(strata_ctx* ctx, int key_bytes, const void* d_a, const int64_t* d_aw, uint64_t na,
    int a_shift, const void* d_b, const int64_t* d_bw, uint64_t nb, int b_shift, int out_shift,
    void* d_out, int64_t* d_out_w, uint64_t out_cap, uint64_t* out_n);

/* The head of a one-atom body (`build_head`, strata-eval/src/naive.rs:526):
 * out[i] = (col(sel_hi) << out_shift) | col(sel_lo) with col 0 = c0 =
 * key >> in_shift, 1 = c1 = the low in_shift bits, 2 = the constant const_hi
 * / const_lo; sel_hi = 3 writes col(sel_lo) alone (a unary head).  A unary
 * input uses in_shift = its key bits (the whole key is c1).  Output keys
 * keep the input order: sort + dedup them for the head relation. */
strata_status strata_op_project(strata_ctx* ctx, int key_bytes_in, const void* d_in, uint64_t n, int in_shift,
    int sel_hi, int sel_lo, uint64_t const_hi, uint64_t const_lo, int key_bytes_out, int out_shift, void* d_out);

/* Aggregate rule  H(G, agg<V>) :- body  (`eval_aggregate_rule` +
 * `fold_aggregate`, strata-eval/src/naive.rs:300-391) over its bindings as
 * sorted keys: the group of a binding is key >> group_shift (group_shift =
 * key bits: one group).  op 0 = count (the number of bindings per group),
 * 1 = sum (wrapping i64), 2 = min, 3 = max of d_vals (one int64 aggregand per
 * binding; unused for count).  Writes the distinct groups ascending to
 * d_groups and their results to d_out (capacity n each); *out_n = groups.
 * Unsorted keys: STRATA_E_CUDA (a bounds status), nothing written. */
strata_status strata_op_aggregate(strata_ctx* ctx, int key_bytes, const void* d_keys, const int64_t* d_vals,
    uint64_t n, int group_shift, int op, void* d_groups, int64_t* d_out, uint64_t* out_n);

/* Merge two sorted, disjoint key runs (with optional int64 weights) into out. */
strata_status strata_op_merge(strata_ctx* ctx, int key_bytes,
    const void* d_a, const int64_t* d_aw, uint64_t na,
    const void* d_b, const int64_t* d_bw, uint64_t nb,
    void* d_out, int64_t* d_out_w);

/* ---- allocation-free sort ---------------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (host callbacks and driver hooks where cudaMalloc is not allowed,
 * embedders whose allocator owns the whole device, latency-critical loops
 * that must not enter the allocator): a stable ascending sort of u32 keys on
 * their low `key_bits` bits (0..32) from d_keys_in into d_keys_out (distinct
 * caller-owned device buffers that must not overlap, else STRATA_E_INVALID;
 * the input is left unchanged), run on `stream`
 * (a cudaStream_t; NULL = the legacy default stream) and finished before the
 * call returns.  It needs no context and calls no allocator: its temporaries
 * live in a fixed 4,483,200-byte array inside the library, which every GPU that
 * loads the library holds until the process exits.  n above
 * STRATA_NOALLOC_SORT_MAX_KEYS returns STRATA_E_INVALID.  The first call on
 * each device looks up the array's device address (once per device, with that
 * device current); make it before any stream capture.  All calls share the
 * array: calls whose GPU work overlaps race and must be serialized by the
 * caller. */
#define STRATA_NOALLOC_SORT_MAX_KEYS (1u << 20)
strata_status strata_sort_u32_noalloc(const uint32_t* d_keys_in, uint32_t* d_keys_out, uint64_t n,
                                      int key_bits, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* STRATA_B200_H */
