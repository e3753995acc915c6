// sk_ops.cuh — host-side entry points of the device operators.  Each function
// launches its kernels on ctx->stream; none synchronizes unless it says so.
#pragma once

#include <stdint.h>

#include "sk_common.cuh"

namespace sk {

// Radix sort limit per call (the onesweep look-back words carry 30-bit counts).
constexpr uint64_t kMaxSortN = (1ull << 30) - 1;
// strata_op_sort and the radix sort itself (64-bit look-back words past kMaxSortN)
constexpr uint64_t kMaxSortKeys = (1ull << 32) - 1;

// Stable LSD radix sort (onesweep) of `n` keys on their low `bits` bits, with
// optional values (V = uint32_t or uint64_t; has_vals selects them).  keys/alt
// (and vals/valt) are a double buffer: on return `*keys` (and `*vals`) point at
// the sorted data and `*alt` at the scratch half.  When `skip_trivial` is set
// the global digit histogram is read back (one synchronization) and passes
// whose digit is constant are skipped.
template <class K, class V>
void radix_sort(strata_ctx* ctx, K** keys, K** alt, V** vals, V** valt, bool has_vals,
                uint64_t n, int bits, bool skip_trivial = true);

// Keys-per-thread choices of the onesweep tile for 4- or 8-byte keys
// (strata_ctx_set_knob); returns how many, writes up to max_out.
int radix_items_choices(int key_bytes, int* out, int max_out);

// Allocation-free u32 key sort on caller-provided scratch (sk_noalloc.cu).
uint64_t radix_sort_u32_static_bytes(uint64_t max_n);
void radix_sort_u32_static(cudaStream_t stream, const uint32_t* in, uint32_t* out, uint64_t n, int bits,
                           unsigned char* scratch, uint64_t max_n, uint32_t* h_status);

// ---- direct-addressed plan (sk_dense.cu) ----
// Index over (c0, c1) in [0, n0) × [0, n1), stored as `rows` rows of `width`
// entries: `colmajor` puts (c0, c1) at c1 * width + c0 (rows by the join
// column of the next round), else at c0 * width + c1.  The width is the
// row's column count rounded up to 32, so no 32-bit word of a bitmap over the
// index spans two rows; the padding entries are never set.
struct DenseLayout {
  int b1;            // key = (c0 << b1) | c1
  uint64_t mask1;    // (1 << b1) - 1
  uint64_t n0, n1;   // column domain sizes
  uint64_t width;    // entries per row (multiple of 32)
  uint64_t rows;     // n1 (colmajor) or n0
  uint64_t entries;  // rows * width
  bool colmajor;
};
DenseLayout dense_layout(int b1, uint64_t n0, uint64_t n1, bool colmajor);
uint64_t dense_tile_size();
uint32_t dense_group_max();
// Group heads of a Δ sorted by join value (see sk_dense.cu): writes hidx
// (Δ row), hpos (exclusive degree prefix, hpos[nh] = total), hseg (CSR
// segment start), hg (group size); out3 = {heads, outputs, candidates}.
// `sums` holds dense_heads_sums(n) words.
template <class K>
void dense_heads(strata_ctx* ctx, const K* dkeys, uint64_t n, int jshift, uint64_t jmask, const uint32_t* off,
                 uint64_t n_nodes, uint64_t* sums, uint32_t* hidx, uint64_t* hpos, uint32_t* hseg, uint8_t* hg,
                 uint64_t* out3);
uint64_t dense_heads_sums(uint64_t n);
// Weight lanes W: int32_t (narrow) or int64_t (wide); Bool uses int32_t and
// ignores it.  D holds WAbs<W> for absent entries.
template <class K, bool TROP, class W = int32_t>
void dense_expand(strata_ctx* ctx, const K* dkeys, const W* dw, uint64_t n_rows, const uint32_t* hidx,
                  const uint64_t* hpos, const uint32_t* hseg, const uint8_t* hg, uint64_t nh, uint64_t total,
                  uint64_t candidates, int pshift, uint64_t pmask, int out_pshift, int out_vshift, const uint32_t* nbr,
                  uint64_t n_nbr, const W* nbr_w, const DenseLayout& lay, uint32_t* bits, W* D,
                  uint32_t* marks, uint64_t* splits_buf);
// The marked entries in index order (keys, Trop weights from D); clears the
// marks.  Used for the bit-row plan's final relation.
template <class K, bool TROP, class W = int32_t>
uint64_t dense_marks_compact(strata_ctx* ctx, uint32_t* marks, const DenseLayout& lay, const W* D, K* out,
                             W* out_w, uint64_t out_cap, uint64_t* states_buf);
uint64_t dense_marks_states(uint64_t entries);
// Heads of the Δ held in `marks` (the entries the last round marked): one
// head per nonzero 32-bit word whose row (join value) has edges, carrying the
// word's bits as its member mask; Trop copies the heads' member weights
// D → Dprev (the values Δ carries through the next round).  Clears marks.
// out4 = {heads, outputs, candidates, Δ tuples}.  `sums` holds
// dense_word_heads_sums(lay) words.
template <bool TROP, class W = int32_t>
void dense_word_heads(strata_ctx* ctx, uint32_t* marks, const DenseLayout& lay, const uint32_t* off,
                      uint64_t n_nodes, uint64_t* sums, uint32_t* hword, uint32_t* hmask, uint64_t* hpos,
                      uint32_t* hseg, const W* D, W* Dprev, uint64_t* out4);
uint64_t dense_word_heads_sums(const DenseLayout& lay);
// One round over word heads: candidates (member, edge) of every head,
// member weights from Dprev; new / improved entries set their marks.
template <bool TROP, class W = int32_t>
void dense_expand_words(strata_ctx* ctx, const uint32_t* hword, const uint32_t* hmask, const uint64_t* hpos,
                        const uint32_t* hseg, uint64_t nh, uint64_t total, uint64_t candidates, uint64_t n_delta,
                        const W* Dprev, int out_pshift, int out_vshift, const uint32_t* nbr, uint64_t n_nbr,
                        const W* nbr_w, const DenseLayout& lay, uint32_t* bits, W* D, uint32_t* marks,
                        uint64_t* splits_buf);
// out[i] = sum of v[0..i) (exclusive) or v[0..i] (inclusive); *total (if
// given, synchronizing) = the sum of all n.
void scan_u64(strata_ctx* ctx, const uint64_t* v, uint64_t n, uint64_t* out, bool inclusive, uint64_t* total);
// In-place exclusive scan of per-tile sums (one block per array); sums[count]
// = total.  `arrays` consecutive arrays of count + 1 words each.
void scan_tile_sums(strata_ctx* ctx, uint64_t* sums, uint64_t count, int arrays = 1);
// Seed the index from keys (and weights); `marks` (optional) marks every
// seeded entry, making the seed the first Δ of the word-head rounds.
template <class K, bool TROP, class W = int32_t>
void dense_seed(strata_ctx* ctx, const K* keys, const W* w, uint64_t n, const DenseLayout& lay, uint32_t* bits,
                W* D, uint32_t* marks);
template <class K, bool TROP, class W = int32_t>
uint64_t dense_compact(strata_ctx* ctx, const uint32_t* bits, const W* D, const DenseLayout& lay, K* out,
                       W* out_w, uint64_t out_cap);

// Exclusive scan of per-element expand degrees (see sk_relops.cu).
// pos[i] = sum_{k<i} deg(i); pos[n] = total.  Returns nothing; read pos[n].
// Grouped mode (gmax > 0): only the first item of each run of equal join
// value (runs split at multiples of gmax) gets its degree; *cand_total (if
// given) receives the sum of every item's degree, i.e. the candidate count.
template <class K>
void expand_offsets(strata_ctx* ctx, const K* dkeys, uint64_t n, int jshift, uint64_t jmask,
                    const uint32_t* off, uint64_t n_nodes, uint64_t* pos, uint32_t gmax = 0,
                    uint64_t* cand_total = nullptr);

// Load-balanced expand: for every Δ tuple i and every CSR neighbour v of its
// join value, emit  out = (kept(i) << out_pshift) | (v << out_vshift), with
// Trop weight w = dw[i] (x) ew[e].  `total` = pos[n].
template <class K, class W, bool TROP>
void expand_emit(strata_ctx* ctx, const K* dkeys, const W* dw, uint64_t n, const uint64_t* pos,
                 uint64_t total, int jshift, uint64_t jmask, int pshift, uint64_t pmask,
                 int out_pshift, int out_vshift, const uint32_t* off, uint64_t n_nodes,
                 const uint32_t* nbr, uint64_t n_nbr, const W* nbr_w, K* out, W* out_w);

// Reduce sorted keys with duplicates to one row per key (Trop: the minimum
// weight).  Writes count to *d_count (device).  `out`/`out_w` capacity >= n.
template <class K, class W, bool TROP>
void reduce_runs(strata_ctx* ctx, const K* keys, const W* w, uint64_t n, K* out, W* out_w,
                 uint64_t* d_count);

// Merge the sorted unique `full` with the sorted unique `cand`:
//   full_out = full ∪ cand (Trop: min weight per key),
//   delta    = keys of cand new to full (Bool) or new / strictly better (Trop).
// d_counts[0] = |full_out|, d_counts[1] = |delta|.
template <class K, class W, bool TROP>
void merge_diff(strata_ctx* ctx, const K* full, const W* full_w, uint64_t nf, const K* cand,
                const W* cand_w, uint64_t nc, K* full_out, W* full_out_w, K* delta, W* delta_w,
                uint64_t* d_counts);

// Plain merge of two sorted disjoint runs.
template <class K, class W, bool TROP>
void merge_disjoint(strata_ctx* ctx, const K* a, const W* aw, uint64_t na, const K* b,
                    const W* bw, uint64_t nb, K* out, W* out_w);

// Dedup + difference against full (operator form): distinct cand keys absent
// from full; Trop: min-reduced keys new to full or strictly better, with the
// better weights also written into full_w.  d_count[0] = output count.
template <class K, class W, bool TROP>
void diff_improve(strata_ctx* ctx, const K* cand, const W* cand_w, uint64_t nc, const K* full,
                  W* full_w, uint64_t nf, K* out, W* out_w, uint64_t* d_count);

// CSR offsets from keys sorted by (join << vbits) | v:
// off[j] = first index with join >= j, for j in [0, n_nodes]; nbr[i] = key & vmask.
template <class K>
void build_csr(strata_ctx* ctx, const K* keys, uint64_t m, int vbits, uint64_t n_nodes,
               uint32_t* off, uint32_t* nbr);

// Count distinct ids below `limit` present in up to three u32 columns.
uint64_t count_distinct_ids(strata_ctx* ctx, const uint32_t* a, uint64_t na, const uint32_t* b,
                            uint64_t nb, const uint32_t* c, uint64_t nc, uint64_t limit);

// max over columns (synchronizing).
uint32_t max_u32(strata_ctx* ctx, const uint32_t* a, uint64_t n);

// Pack two u32 columns into keys (c0 << shift) | c1, optional weight conversion
// from (int64 w, u8 inf) to W codes (inf -> WInf<W>, finite v -> v - ctx->wshift).
// Sets ST_SENTINEL when a finite weight has no code.
template <class K, class W, bool TROP>
void pack_pairs(strata_ctx* ctx, const uint32_t* c0, const uint32_t* c1, const int64_t* w,
                const uint8_t* inf, uint64_t n, int shift, K* keys, W* ow);

// Unpack keys to columns (and W codes to int64 values + inf mask, adding
// ctx->wshift to finite codes).
template <class K, class W, bool TROP>
void unpack_pairs(strata_ctx* ctx, const K* keys, const W* w, uint64_t n, int shift,
                  uint32_t* c0, uint32_t* c1, int64_t* ow, uint8_t* oinf);

// Min and max finite weight over (w, inf) columns (synchronizing); false when
// there is none (both 0).  NULL w: every weight is Finite(0).
bool weight_range(strata_ctx* ctx, const int64_t* w, const uint8_t* inf, uint64_t n, int64_t* mn, int64_t* mx);

// Max |finite weight| over (w, inf) columns (synchronizing); 0 when n == 0.
uint64_t max_abs_weight(strata_ctx* ctx, const int64_t* w, const uint8_t* inf, uint64_t n);

// Order-independent fingerprint of (keys, weight values = codes + ctx->wshift).
template <class K, class W, bool TROP>
uint64_t fingerprint(strata_ctx* ctx, const K* keys, const W* w, uint64_t n, int shift);

// ---- operator surface (sk_opsurf.cu) ----
// One binary body  h(X,Z) :- a(X,Y), b(Y,Z):  a = (X << d_shift) | Y (any
// order), b = (Y << r_shift) | Z sorted ascending; output (X << out_shift) | Z
// with ⊗ weights (Trop when dw != NULL; int64, INT64_MAX = +inf) in a's
// order.  Returns the binding count; writes only when out != NULL and
// out_cap >= count (*written says whether it did).
template <class K>
uint64_t op_join(strata_ctx* ctx, const K* dk, const int64_t* dw, uint64_t nd, int d_shift, const K* rk,
                 const int64_t* rw, uint64_t nr, int r_shift, int out_shift, K* out, int64_t* out_w, uint64_t out_cap,
                 bool* written);
// out[i] = (col(sel_hi) << out_shift) | col(sel_lo), col 0 = c0, 1 = c1,
// 2 = the constant; sel_hi 3 = a one-column output (col(sel_lo) alone).
template <class KI, class KO>
void op_project(strata_ctx* ctx, const KI* in, uint64_t n, int in_shift, int sel_hi, int sel_lo, uint64_t const_hi,
                uint64_t const_lo, int out_shift, KO* out);
// Rows with c0 == c1 (mode 0), c0 == k (1) or c1 == k (2), in input order.
template <class K>
uint64_t op_select(strata_ctx* ctx, const K* keys, const int64_t* w, uint64_t n, int shift, int mode, uint64_t k,
                   K* out, int64_t* out_w);
// Rows of a whose key is in the sorted b; Trop: weight a.w ⊗ b.w.
template <class K>
uint64_t op_intersect(strata_ctx* ctx, const K* a, const int64_t* aw, uint64_t na, const K* b, const int64_t* bw,
                      uint64_t nb, K* out, int64_t* out_w);
// Rows whose probe key (NULL: the row key) is in (anti: absent from) sorted b.
template <class K>
uint64_t op_semijoin(strata_ctx* ctx, const K* rows, const int64_t* w, uint64_t n, const K* probe, const K* b,
                     uint64_t nb, bool anti, K* out, int64_t* out_w);
// Groups key >> gshift of sorted keys with count / sum / min / max (op 0..3)
// of vals; returns the number of groups.
template <class K>
uint64_t op_aggregate(strata_ctx* ctx, const K* keys, const int64_t* vals, uint64_t n, int gshift, int op, K* groups,
                      int64_t* out_vals);

// ---- ASP grounding-simplify filter (sk_asp.cu) ----
struct AspResult {
  uint64_t n_rules = 0;
  int32_t* head = nullptr;        // malloc'd, n_rules
  uint32_t* body_start = nullptr;  // malloc'd, n_rules + 1
  int32_t* body_lit = nullptr;     // malloc'd, body_start[n_rules]
};
AspResult asp_simplify(strata_ctx* ctx, uint64_t n_rules, const int32_t* head, const uint32_t* bstart,
                       const int32_t* lit, uint64_t n_atoms, const uint8_t* poss, const uint8_t* cert);

// ---- text input / output (sk_text.cu) ----
// One Soufflé TSV load: rows of `arity` symbol cells (+ a trailing i64 weight
// when trop), interned first-seen after the n_dict dictionary strings.  On a
// bad row err_kind = 1 (cell count), 2 (empty symbol cell err_col) or 3
// (weight) with its 1-based line; else cols (column-major, rows x arity),
// w, and the new symbols (n_new strings in id order, bytes + offsets), all
// malloc'd for the caller.
struct TsvResult {
  uint64_t rows = 0;
  uint32_t* cols = nullptr;
  int64_t* w = nullptr;
  uint64_t n_new = 0;
  char* new_bytes = nullptr;
  uint64_t* new_off = nullptr;
  uint64_t err_line = 0;
  uint32_t err_col = 0;
  int err_kind = 0;
};
TsvResult tsv_load(strata_ctx* ctx, const char* text, uint64_t text_len, uint32_t arity, bool trop,
                   const char* dict_bytes, const uint64_t* dict_off, uint64_t n_dict);
// The canonical text of a binary relation handle (malloc'd, NUL-terminated);
// returns its length.
uint64_t render_rel(strata_ctx* ctx, const strata_rel* rel, const char* name, const char* dict_bytes,
                    const uint64_t* dict_off, uint64_t n_dict, char** out_text);

}  // namespace sk
